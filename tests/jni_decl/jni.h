/* Declarations of the JNI types and JNIEnv calls that B200FemJNI.cc uses,
   for compile-checking the shim where no JDK is installed.  Only the names
   and signatures matter here; the object built from them is a syntax and
   type check and is never loaded by a JVM (a real build uses the JDK's
   jni.h). */
#ifndef B200FEM_TEST_JNI_DECL_H
#define B200FEM_TEST_JNI_DECL_H
#include <stdint.h>
typedef int32_t jint;
typedef int64_t jlong;
typedef double jdouble;
typedef uint8_t jboolean;
typedef jint jsize;
class _jobject {};
typedef _jobject* jobject;
typedef jobject jclass;
typedef jobject jstring;
typedef jobject jarray;
typedef jarray jdoubleArray;
typedef jarray jintArray;
typedef jarray jlongArray;
#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL
#define JNI_COMMIT 1
#define JNI_ABORT 2
struct JNIEnv {
  jsize GetArrayLength(jarray a);
  jdouble* GetDoubleArrayElements(jdoubleArray a, jboolean* isCopy);
  void ReleaseDoubleArrayElements(jdoubleArray a, jdouble* p, jint mode);
  jint* GetIntArrayElements(jintArray a, jboolean* isCopy);
  void ReleaseIntArrayElements(jintArray a, jint* p, jint mode);
  void SetDoubleArrayRegion(jdoubleArray a, jsize start, jsize len, const jdouble* buf);
  void SetIntArrayRegion(jintArray a, jsize start, jsize len, const jint* buf);
  void SetLongArrayRegion(jlongArray a, jsize start, jsize len, const jlong* buf);
  jstring NewStringUTF(const char* s);
};
#endif
