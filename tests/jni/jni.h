/*
 * TEST FIXTURE: a minimal jni.h for compiling the JNI bridge (tdp1375_b200/csrc/jni_bridge.cpp)
 * without a JDK.  It declares the JNI types, macros and the JNIEnv member functions the
 * bridge calls, with the names, argument lists and meaning of the Java Native Interface
 * specification (chapter 4, "JNI Functions").  The function table is this file's own: it
 * lists only those functions and does not reproduce the JDK's table layout, so objects
 * built against it work only with tests/jni/fake_jvm.cpp, which fills the table.
 */
#ifndef TDP_TEST_JNI_H
#define TDP_TEST_JNI_H

#include <stdint.h>

typedef int8_t jbyte;
typedef uint8_t jboolean;
typedef int32_t jint;
typedef int64_t jlong;
typedef float jfloat;
typedef jint jsize;

class _jobject {};
class _jclass : public _jobject {};
class _jthrowable : public _jobject {};
class _jstring : public _jobject {};
class _jarray : public _jobject {};
class _jbyteArray : public _jarray {};
class _jintArray : public _jarray {};
class _jobjectArray : public _jarray {};
typedef _jobject *jobject;
typedef _jclass *jclass;
typedef _jthrowable *jthrowable;
typedef _jarray *jarray;
typedef _jbyteArray *jbyteArray;
typedef _jintArray *jintArray;
typedef _jobjectArray *jobjectArray;

#define JNI_FALSE 0
#define JNI_TRUE 1
#define JNI_OK 0
#define JNI_COMMIT 1 /* ReleasePrimitiveArrayCritical mode: copy back, keep the buffer */
#define JNI_ABORT 2  /* ReleasePrimitiveArrayCritical mode: free the buffer, no copy back */

#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL

struct JNIEnv_;

struct TdpTestJniFunctions {
    jboolean (*ExceptionCheck)(JNIEnv_ *env);
    void (*ExceptionClear)(JNIEnv_ *env);
    jclass (*FindClass)(JNIEnv_ *env, const char *name);
    jint (*ThrowNew)(JNIEnv_ *env, jclass cls, const char *message);
    void (*DeleteLocalRef)(JNIEnv_ *env, jobject ref);
    jsize (*GetArrayLength)(JNIEnv_ *env, jarray array);
    void *(*GetPrimitiveArrayCritical)(JNIEnv_ *env, jarray array, jboolean *isCopy);
    void (*ReleasePrimitiveArrayCritical)(JNIEnv_ *env, jarray array, void *carray, jint mode);
    jobjectArray (*NewObjectArray)(JNIEnv_ *env, jsize length, jclass elementClass, jobject initialElement);
    void (*SetObjectArrayElement)(JNIEnv_ *env, jobjectArray array, jsize index, jobject value);
    jintArray (*NewIntArray)(JNIEnv_ *env, jsize length);
    void (*SetIntArrayRegion)(JNIEnv_ *env, jintArray array, jsize start, jsize len, const jint *buf);
    jbyteArray (*NewByteArray)(JNIEnv_ *env, jsize length);
    void (*SetByteArrayRegion)(JNIEnv_ *env, jbyteArray array, jsize start, jsize len, const jbyte *buf);
};

struct JNIEnv_ {
    const TdpTestJniFunctions *functions;
    jboolean ExceptionCheck() { return functions->ExceptionCheck(this); }
    void ExceptionClear() { functions->ExceptionClear(this); }
    jclass FindClass(const char *name) { return functions->FindClass(this, name); }
    jint ThrowNew(jclass cls, const char *message) { return functions->ThrowNew(this, cls, message); }
    void DeleteLocalRef(jobject ref) { functions->DeleteLocalRef(this, ref); }
    jsize GetArrayLength(jarray array) { return functions->GetArrayLength(this, array); }
    void *GetPrimitiveArrayCritical(jarray array, jboolean *isCopy) {
        return functions->GetPrimitiveArrayCritical(this, array, isCopy);
    }
    void ReleasePrimitiveArrayCritical(jarray array, void *carray, jint mode) {
        functions->ReleasePrimitiveArrayCritical(this, array, carray, mode);
    }
    jobjectArray NewObjectArray(jsize length, jclass elementClass, jobject initialElement) {
        return functions->NewObjectArray(this, length, elementClass, initialElement);
    }
    void SetObjectArrayElement(jobjectArray array, jsize index, jobject value) {
        functions->SetObjectArrayElement(this, array, index, value);
    }
    jintArray NewIntArray(jsize length) { return functions->NewIntArray(this, length); }
    void SetIntArrayRegion(jintArray array, jsize start, jsize len, const jint *buf) {
        functions->SetIntArrayRegion(this, array, start, len, buf);
    }
    jbyteArray NewByteArray(jsize length) { return functions->NewByteArray(this, length); }
    void SetByteArrayRegion(jbyteArray array, jsize start, jsize len, const jbyte *buf) {
        functions->SetByteArrayRegion(this, array, start, len, buf);
    }
};
typedef JNIEnv_ JNIEnv;

#endif /* TDP_TEST_JNI_H */
