/*
 * cumf_jni.h -- the Spark JNI symbols exported by libGPUALS.so.
 *
 * Same Java class, method names and signatures as the reference's javah header
 * als/src/org_apache_spark_ml_recommendation_CuMFJNIInterface.h:29-40, so
 * Spark's CuMFJNIInterface (loaded from spark.mllib.ALS.useGPU) binds to this
 * library unchanged. The JNI types are declared here from the JNI
 * specification so the library builds without a JDK; a JVM passes its own
 * JNIEnv, whose function table this code indexes per that specification.
 */
#ifndef CUMF_JNI_H_
#define CUMF_JNI_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t jint;
typedef double jdouble;
typedef float jfloat;
typedef void *jobject;
typedef jobject jobjectArray;
typedef jobject jintArray;
typedef jobject jfloatArray;
typedef jobject jclass;
typedef jobject jarray;
typedef jint jsize;
typedef uint8_t jboolean;
/* A JNIEnv* points at a pointer to the JNI function table. */
typedef const void *const *JNIEnv_table;
typedef JNIEnv_table JNIEnv_;

/* Method doALSWithCSR, signature (IIIID[[[F[I[I[F)[[F (reference header :31-32,
 * body als/src/CuMFJNIInterface.cpp:25-132). Returns float[m][f], or NULL
 * after printing the error (the reference falls off the end of the function
 * in that case). */
jobjectArray Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR(
    JNIEnv_ *env, jobject obj, jint m, jint n, jint f, jint nnz, jdouble lambda,
    jobjectArray sortedSrcFactors, jintArray csrRow, jintArray csrCol, jfloatArray csrVal);

/* Method testjni, signature ()V (reference header :39-40, body CuMFJNIInterface.cpp:134-138). */
void Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_testjni(JNIEnv_ *env, jobject obj);

#ifdef __cplusplus
}
#endif
#endif /* CUMF_JNI_H_ */
