// Spark JNI entry of libGPUALS.so: marshals Spark's factor blocks and CSR
// arrays into native memory, runs the drop-in doALSWithCSR half-step, and
// returns float[m][f]. Behaviour follows als/src/CuMFJNIInterface.cpp:25-132:
// device chosen round-robin per call, one stream per call, source factors
// flattened in block order, CSR uploaded to mallocBest memory that the
// half-step frees.
//
// JNI functions are reached through the JNIEnv function table by the slot
// numbers of the JNI specification's interface function table, so no JDK
// header is needed to build.
#include <cuda_runtime.h>
#include <thrust/system/cuda/error.h>
#include <thrust/system_error.h>

#include <cstdio>
#include <cstring>

#include "../../include/als_b200.h"
#include "../../include/cumf_jni.h"

namespace {

// Slots of the JNI interface function table (JNI specification, chapter 4).
enum JniSlot {
  kFindClass = 6,
  kDeleteLocalRef = 23,
  kGetArrayLength = 171,
  kNewObjectArray = 172,
  kGetObjectArrayElement = 173,
  kSetObjectArrayElement = 174,
  kNewFloatArray = 181,
  kSetFloatArrayRegion = 213,
  kGetPrimitiveArrayCritical = 222,
  kReleasePrimitiveArrayCritical = 223,
};

template <typename Fn>
Fn slot(JNIEnv_ *env, int idx) {
  const void *const *table = *env;
  return reinterpret_cast<Fn>(const_cast<void *>(table[idx]));
}

struct Jni {
  JNIEnv_ *env;
  jclass FindClass(const char *name) {
    return slot<jclass (*)(JNIEnv_ *, const char *)>(env, kFindClass)(env, name);
  }
  void DeleteLocalRef(jobject o) {
    slot<void (*)(JNIEnv_ *, jobject)>(env, kDeleteLocalRef)(env, o);
  }
  jsize GetArrayLength(jarray a) {
    return slot<jsize (*)(JNIEnv_ *, jarray)>(env, kGetArrayLength)(env, a);
  }
  jobjectArray NewObjectArray(jsize len, jclass cls, jobject init) {
    return slot<jobjectArray (*)(JNIEnv_ *, jsize, jclass, jobject)>(env, kNewObjectArray)(
        env, len, cls, init);
  }
  jobject GetObjectArrayElement(jobjectArray a, jsize i) {
    return slot<jobject (*)(JNIEnv_ *, jobjectArray, jsize)>(env, kGetObjectArrayElement)(env, a, i);
  }
  void SetObjectArrayElement(jobjectArray a, jsize i, jobject v) {
    slot<void (*)(JNIEnv_ *, jobjectArray, jsize, jobject)>(env, kSetObjectArrayElement)(env, a, i, v);
  }
  jfloatArray NewFloatArray(jsize len) {
    return slot<jfloatArray (*)(JNIEnv_ *, jsize)>(env, kNewFloatArray)(env, len);
  }
  void SetFloatArrayRegion(jfloatArray a, jsize start, jsize len, const jfloat *buf) {
    slot<void (*)(JNIEnv_ *, jfloatArray, jsize, jsize, const jfloat *)>(env, kSetFloatArrayRegion)(
        env, a, start, len, buf);
  }
  void *GetPrimitiveArrayCritical(jarray a, jboolean *copy) {
    return slot<void *(*)(JNIEnv_ *, jarray, jboolean *)>(env, kGetPrimitiveArrayCritical)(env, a, copy);
  }
  void ReleasePrimitiveArrayCritical(jarray a, void *p, jint mode) {
    slot<void (*)(JNIEnv_ *, jarray, void *, jint)>(env, kReleasePrimitiveArrayCritical)(env, a, p, mode);
  }
};

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw thrust::system_error(e, thrust::cuda_category(), what);
}

}  // namespace

extern "C" jobjectArray Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR(
    JNIEnv_ *env, jobject, jint m, jint n, jint f, jint nnz, jdouble lambda,
    jobjectArray sortedSrcFactors, jintArray csrRow, jintArray csrCol, jfloatArray csrVal) {
  Jni J{env};
  float *thetaTHost = nullptr, *XTHost = nullptr;
  cudaStream_t stream = nullptr;
  try {
    const int dev = get_gpu();
    if (dev < 0) throw thrust::system_error(cudaErrorNoDevice, thrust::cuda_category(), "no GPU");
    check(cudaSetDevice(dev), "cudaSetDevice");
    check(cudaStreamCreate(&stream), "cudaStreamCreate");
    check(cudaMallocHost((void **)&thetaTHost, sizeof(float) * (size_t)n * f), "pinned theta");
    check(cudaMallocHost((void **)&XTHost, sizeof(float) * (size_t)m * f), "pinned X");
    // Flatten the sorted source factor blocks: float[blocks][factors][f].
    const jsize blocks = J.GetArrayLength(sortedSrcFactors);
    size_t index = 0;
    for (jsize b = 0; b < blocks; ++b) {
      jobjectArray blk = (jobjectArray)J.GetObjectArrayElement(sortedSrcFactors, b);
      const jsize count = J.GetArrayLength(blk);
      for (jsize j = 0; j < count; ++j) {
        jfloatArray fac = (jfloatArray)J.GetObjectArrayElement(blk, j);
        if (index < (size_t)n) {
          float *p = (float *)J.GetPrimitiveArrayCritical(fac, nullptr);
          std::memcpy(thetaTHost + index * f, p, sizeof(float) * f);
          J.ReleasePrimitiveArrayCritical(fac, p, 0);
        }
        ++index;
        J.DeleteLocalRef(fac);
      }
      J.DeleteLocalRef(blk);
    }
    if (index != (size_t)n)
      throw thrust::system_error(cudaErrorInvalidValue, thrust::cuda_category(),
                                 "source factor count differs from n");
    // The CSR arrays go to doALSWithCSR, which frees them; until then they
    // are this call's, and a failure before the hand-over frees them here.
    struct CsrArrays {
      int *row = nullptr, *col = nullptr;
      float *val = nullptr;
      bool handed_over = false;
      ~CsrArrays() {
        if (handed_over) return;
        freeBest(row);
        freeBest(col);
        freeBest(val);
      }
    } csr;
    check(mallocBest((void **)&csr.row, sizeof(int) * ((size_t)m + 1)), "mallocBest row");
    check(mallocBest((void **)&csr.col, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)), "mallocBest col");
    check(mallocBest((void **)&csr.val, sizeof(float) * (size_t)(nnz > 0 ? nnz : 1)), "mallocBest val");
    int *d_row = csr.row, *d_col = csr.col;
    float *d_val = csr.val;
    void *hr = J.GetPrimitiveArrayCritical(csrRow, nullptr);
    void *hc = J.GetPrimitiveArrayCritical(csrCol, nullptr);
    void *hv = J.GetPrimitiveArrayCritical(csrVal, nullptr);
    cudaError_t e = cudaMemcpyAsync(d_row, hr, sizeof(int) * ((size_t)m + 1), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && nnz > 0)
      e = cudaMemcpyAsync(d_col, hc, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && nnz > 0)
      e = cudaMemcpyAsync(d_val, hv, sizeof(float) * (size_t)nnz, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    J.ReleasePrimitiveArrayCritical(csrRow, hr, 0);
    J.ReleasePrimitiveArrayCritical(csrCol, hc, 0);
    J.ReleasePrimitiveArrayCritical(csrVal, hv, 0);
    check(e, "CSR upload");
    csr.handed_over = true;  // doALSWithCSR frees them, on success and on failure
    doALSWithCSR(stream, d_row, d_col, d_val, thetaTHost, XTHost, m, n, f, nnz, (float)lambda, 1);
    jclass floatArrayClass = J.FindClass("[F");
    jobjectArray output = J.NewObjectArray(m, floatArrayClass, nullptr);
    for (jint i = 0; i < m; ++i) {
      jfloatArray row = J.NewFloatArray(f);
      J.SetFloatArrayRegion(row, 0, f, XTHost + (size_t)i * f);
      J.SetObjectArrayElement(output, i, row);
      J.DeleteLocalRef(row);
    }
    cudaFreeHost(thetaTHost);
    cudaFreeHost(XTHost);
    check(cudaStreamSynchronize(stream), "sync");
    check(cudaStreamDestroy(stream), "stream destroy");
    return output;
  } catch (thrust::system_error &err) {
    std::printf("CUDA error during some function: %s", err.what());
    if (thetaTHost) cudaFreeHost(thetaTHost);
    if (XTHost) cudaFreeHost(XTHost);
    if (stream) cudaStreamDestroy(stream);
    return nullptr;
  }
}

extern "C" void Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_testjni(JNIEnv_ *, jobject) {
  std::printf("*******in native code of testjni ...\n");
}
