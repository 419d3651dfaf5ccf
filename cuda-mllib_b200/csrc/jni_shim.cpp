// Spark JNI entry of libGPUALS.so: marshals Spark's factor blocks into
// native memory, runs the drop-in half-step on the CSR arrays, and returns
// float[m][f]. Behaviour follows als/src/CuMFJNIInterface.cpp:25-132: device
// chosen round-robin per call, source factors flattened in block order, the
// half-step of doALSWithCSR (same options and result), the result returned as
// one float[f] per row.
//
// Per-call costs of the reference that this shim does not pay:
//  - it uploads the whole CSR into mallocBest memory (:93-118) and only then
//    starts the half-step, which uploads theta, solves and downloads X, one
//    step after the other. Here als_half_step_host uploads the ratings in row
//    ranges and solves each range while the next one crosses PCIe;
//  - it pins fresh host buffers for theta and X on every call (cudaMallocHost,
//    CuMFJNIInterface.cpp:53-57; page-locking 192 MB takes tens of ms) and
//    creates and destroys a stream (:32-34). Here both are leased from
//    per-device pools kept across calls (concurrent Spark tasks each get their
//    own), and the device buffers come from the library's block cache;
//  - it makes five JNI calls per source factor (:64-76: element, critical
//    section, memcpy, release, delete). Here each factor is one
//    GetObjectArrayElement and one GetFloatArrayRegion straight into the
//    pinned buffer, with local references released a frame of 256 at a time,
//    and the result rows are built the same way.
// The factor values themselves are sent again by Spark on every call (a
// destination block's source factors are a different selection each time)
// and are uploaded again: recognising an unchanged 192 MB block would cost
// more host time than its upload from pinned memory.
//
// JNI functions are reached through the JNIEnv function table by the slot
// numbers of the JNI specification's interface function table, so no JDK
// header is needed to build.
#include <cuda_runtime.h>
#include <thrust/system/cuda/error.h>
#include <thrust/system_error.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/als_b200.h"
#include "../../include/cumf_jni.h"

namespace {

// Slots of the JNI interface function table (JNI specification, chapter 4).
enum JniSlot {
  kFindClass = 6,
  kPushLocalFrame = 19,
  kPopLocalFrame = 20,
  kDeleteLocalRef = 23,
  kGetArrayLength = 171,
  kNewObjectArray = 172,
  kGetObjectArrayElement = 173,
  kSetObjectArrayElement = 174,
  kNewFloatArray = 181,
  kGetFloatArrayRegion = 205,
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
  jint PushLocalFrame(jint capacity) {
    return slot<jint (*)(JNIEnv_ *, jint)>(env, kPushLocalFrame)(env, capacity);
  }
  jobject PopLocalFrame(jobject result) {
    return slot<jobject (*)(JNIEnv_ *, jobject)>(env, kPopLocalFrame)(env, result);
  }
  void GetFloatArrayRegion(jfloatArray a, jsize start, jsize len, jfloat *buf) {
    slot<void (*)(JNIEnv_ *, jfloatArray, jsize, jsize, jfloat *)>(env, kGetFloatArrayRegion)(
        env, a, start, len, buf);
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

constexpr int kFrame = 256;            // local references per JNI frame
constexpr size_t kPinnedMax = 8ull << 30;  // idle pinned bytes kept per device
constexpr int kDevices = 64;

// Pinned host buffers and streams of one device, kept across calls.
struct DevicePools {
  std::mutex mu;
  std::vector<std::pair<size_t, float *>> idle_bufs;  // (capacity in floats, buffer)
  size_t idle_bytes = 0;
  std::vector<cudaStream_t> idle_streams;
};
DevicePools &pools(int dev) {
  static DevicePools *p = new DevicePools[kDevices];  // never destroyed (see als_api.cu)
  return p[dev];
}

// A pinned buffer of at least `floats` floats, leased for one call.
struct PinnedLease {
  int dev;
  float *p = nullptr;
  size_t cap = 0;
  PinnedLease(int d, size_t floats) : dev(d) {
    DevicePools &P = pools(dev);
    {
      std::lock_guard<std::mutex> lk(P.mu);
      auto best = P.idle_bufs.end();
      for (auto it = P.idle_bufs.begin(); it != P.idle_bufs.end(); ++it)
        if (it->first >= floats && (best == P.idle_bufs.end() || it->first < best->first)) best = it;
      if (best != P.idle_bufs.end()) {
        cap = best->first;
        p = best->second;
        P.idle_bytes -= cap * sizeof(float);
        P.idle_bufs.erase(best);
        return;
      }
    }
    cap = std::max<size_t>(floats + floats / 8, 1024);
    check(cudaMallocHost((void **)&p, cap * sizeof(float)), "pinned buffer");
  }
  ~PinnedLease() {
    if (!p) return;
    DevicePools &P = pools(dev);
    std::lock_guard<std::mutex> lk(P.mu);
    P.idle_bufs.push_back({cap, p});
    P.idle_bytes += cap * sizeof(float);
    while (P.idle_bytes > kPinnedMax && !P.idle_bufs.empty()) {
      auto big = std::max_element(P.idle_bufs.begin(), P.idle_bufs.end());
      cudaFreeHost(big->second);
      P.idle_bytes -= big->first * sizeof(float);
      P.idle_bufs.erase(big);
    }
  }
};

// A stream of the device, leased for one call. A call that failed may have
// left work queued: its stream is synchronised before it is reused.
struct StreamLease {
  int dev;
  cudaStream_t s = nullptr;
  explicit StreamLease(int d) : dev(d) {
    DevicePools &P = pools(dev);
    {
      std::lock_guard<std::mutex> lk(P.mu);
      if (!P.idle_streams.empty()) {
        s = P.idle_streams.back();
        P.idle_streams.pop_back();
        return;
      }
    }
    check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
  }
  ~StreamLease() {
    if (!s) return;
    if (cudaStreamSynchronize(s) != cudaSuccess) {  // a broken stream is not reused
      cudaGetLastError();
      cudaStreamDestroy(s);
      return;
    }
    DevicePools &P = pools(dev);
    std::lock_guard<std::mutex> lk(P.mu);
    P.idle_streams.push_back(s);
  }
};

}  // namespace

extern "C" jobjectArray Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR(
    JNIEnv_ *env, jobject, jint m, jint n, jint f, jint nnz, jdouble lambda,
    jobjectArray sortedSrcFactors, jintArray csrRow, jintArray csrCol, jfloatArray csrVal) {
  Jni J{env};
  try {
    const int dev = get_gpu();
    if (dev < 0) throw thrust::system_error(cudaErrorNoDevice, thrust::cuda_category(), "no GPU");
    if (dev >= kDevices || m < 0 || n < 0 || f <= 0 || nnz < 0)
      throw thrust::system_error(cudaErrorInvalidValue, thrust::cuda_category(), "bad sizes");
    check(cudaSetDevice(dev), "cudaSetDevice");
    StreamLease stream(dev);
    PinnedLease theta(dev, (size_t)n * f), X(dev, (size_t)m * f);
    float *thetaTHost = theta.p, *XTHost = X.p;
    // Flatten the sorted source factor blocks, float[blocks][factors][f],
    // straight into the pinned buffer.
    const jsize blocks = J.GetArrayLength(sortedSrcFactors);
    size_t index = 0;
    for (jsize b = 0; b < blocks; ++b) {
      jobjectArray blk = (jobjectArray)J.GetObjectArrayElement(sortedSrcFactors, b);
      const jsize count = J.GetArrayLength(blk);
      for (jsize j0 = 0; j0 < count; j0 += kFrame) {
        if (J.PushLocalFrame(kFrame) != 0)
          throw thrust::system_error(cudaErrorMemoryAllocation, thrust::cuda_category(), "JNI frame");
        const jsize j1 = std::min<jsize>(count, j0 + kFrame);
        for (jsize j = j0; j < j1; ++j, ++index) {
          if (index >= (size_t)n) continue;
          jfloatArray fac = (jfloatArray)J.GetObjectArrayElement(blk, j);
          J.GetFloatArrayRegion(fac, 0, f, thetaTHost + index * f);
        }
        J.PopLocalFrame(nullptr);
      }
      J.DeleteLocalRef(blk);
    }
    if (index != (size_t)n)
      throw thrust::system_error(cudaErrorInvalidValue, thrust::cuda_category(),
                                 "source factor count differs from n");
    // The CSR arrays go straight from the Java arrays to the pipelined
    // half-step (ranges of ratings uploaded while the previous range is
    // solved), which reads them and leaves them to the caller.
    void *hr = J.GetPrimitiveArrayCritical(csrRow, nullptr);
    void *hc = J.GetPrimitiveArrayCritical(csrCol, nullptr);
    void *hv = J.GetPrimitiveArrayCritical(csrVal, nullptr);
    int rc = ALS_ERR_INVALID;
    const char *why = "the JVM gave no access to the CSR arrays";
    if (hr && hc && hv) {
      rc = als_half_step_host(stream.s, static_cast<const int *>(hr), static_cast<const int *>(hc),
                              static_cast<const float *>(hv), thetaTHost, XTHost, m, n, f, nnz,
                              (float)lambda, 0);
      why = nullptr;
    }
    if (hv) J.ReleasePrimitiveArrayCritical(csrVal, hv, 0);
    if (hc) J.ReleasePrimitiveArrayCritical(csrCol, hc, 0);
    if (hr) J.ReleasePrimitiveArrayCritical(csrRow, hr, 0);
    if (rc != ALS_OK)
      throw thrust::system_error(rc == ALS_ERR_INVALID ? cudaErrorInvalidValue : cudaErrorLaunchFailure,
                                 thrust::cuda_category(), why ? why : als_last_error());
    // float[m][f], a frame of rows at a time
    jclass floatArrayClass = J.FindClass("[F");
    jobjectArray output = J.NewObjectArray(m, floatArrayClass, nullptr);
    if (!output) return nullptr;  // the JVM's OutOfMemoryError is pending
    for (jint i0 = 0; i0 < m; i0 += kFrame) {
      if (J.PushLocalFrame(kFrame) != 0) return nullptr;
      const jint i1 = std::min<jint>(m, i0 + kFrame);
      for (jint i = i0; i < i1; ++i) {
        jfloatArray row = J.NewFloatArray(f);
        if (!row) {
          J.PopLocalFrame(nullptr);
          return nullptr;
        }
        J.SetFloatArrayRegion(row, 0, f, XTHost + (size_t)i * f);
        J.SetObjectArrayElement(output, i, row);
      }
      J.PopLocalFrame(nullptr);
    }
    return output;
  } catch (thrust::system_error &err) {
    std::printf("CUDA error during some function: %s", err.what());
    return nullptr;
  }
}

extern "C" void Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_testjni(JNIEnv_ *, jobject) {
  std::printf("*******in native code of testjni ...\n");
}
