/*
 * Declarations-only JNI header for building the engine's JNI layer where no JDK is installed.
 *
 * It declares what the layer uses of the Java Native Interface as the JNI specification defines it: the primitive
 * and reference types, and the function table an env points to.  A JNIEnv is a pointer to the function table (the
 * C binding of the specification; the C++ binding wraps the same pointer), and each function sits at the index the
 * specification's "Interface Function Table" gives it, so a library built against this header calls a real JVM's
 * functions correctly.  Only the entries the layer calls are named (olfjni_* helpers below); the others are plain
 * slots.
 */
#ifndef OLF_JNI_STUB_H
#define OLF_JNI_STUB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t jint;
typedef int64_t jlong;
typedef int8_t jbyte;
typedef uint8_t jboolean;
typedef uint16_t jchar;
typedef int16_t jshort;
typedef float jfloat;
typedef double jdouble;
typedef jint jsize;

struct _jobject;
typedef struct _jobject* jobject;
typedef jobject jclass;
typedef jobject jthrowable;
typedef jobject jstring;
typedef jobject jarray;
typedef jarray jbooleanArray;
typedef jarray jbyteArray;
typedef jarray jcharArray;
typedef jarray jshortArray;
typedef jarray jintArray;
typedef jarray jlongArray;
typedef jarray jfloatArray;
typedef jarray jdoubleArray;
typedef jarray jobjectArray;

#define JNI_FALSE 0
#define JNI_TRUE 1
#define JNI_ABORT 2

#define JNIEXPORT __attribute__((visibility("default")))
#define JNIIMPORT
#define JNICALL

/* The function table: 235 slots (up to the JDK 21 additions). */
struct JNINativeInterface_ {
    void* slot[235];
};
typedef const struct JNINativeInterface_* JNIEnv;

/* Slot indices of the functions the layer calls (JNI specification, Interface Function Table). */
enum {
    OLFJNI_FIND_CLASS = 6,
    OLFJNI_THROW_NEW = 14,
    OLFJNI_EXCEPTION_CLEAR = 17,
    OLFJNI_DELETE_LOCAL_REF = 23,
    OLFJNI_GET_ARRAY_LENGTH = 171,
    OLFJNI_NEW_OBJECT_ARRAY = 172,
    OLFJNI_GET_OBJECT_ARRAY_ELEMENT = 173,
    OLFJNI_SET_OBJECT_ARRAY_ELEMENT = 174,
    OLFJNI_NEW_INT_ARRAY = 179,
    OLFJNI_NEW_DOUBLE_ARRAY = 182,
    OLFJNI_GET_BOOLEAN_ARRAY_REGION = 199,
    OLFJNI_GET_BYTE_ARRAY_REGION = 200,
    OLFJNI_GET_INT_ARRAY_REGION = 203,
    OLFJNI_GET_DOUBLE_ARRAY_REGION = 206,
    OLFJNI_SET_INT_ARRAY_REGION = 211,
    OLFJNI_SET_DOUBLE_ARRAY_REGION = 214,
    OLFJNI_EXCEPTION_CHECK = 228
};

#define OLFJNI_FN(env, idx, type) ((type)((*(env))->slot[idx]))

static inline jclass olfjni_FindClass(JNIEnv* env, const char* name) {
    return OLFJNI_FN(env, OLFJNI_FIND_CLASS, jclass (*)(JNIEnv*, const char*))(env, name);
}
static inline jint olfjni_ThrowNew(JNIEnv* env, jclass cls, const char* msg) {
    return OLFJNI_FN(env, OLFJNI_THROW_NEW, jint (*)(JNIEnv*, jclass, const char*))(env, cls, msg);
}
static inline void olfjni_DeleteLocalRef(JNIEnv* env, jobject o) {
    OLFJNI_FN(env, OLFJNI_DELETE_LOCAL_REF, void (*)(JNIEnv*, jobject))(env, o);
}
static inline jsize olfjni_GetArrayLength(JNIEnv* env, jarray a) {
    return OLFJNI_FN(env, OLFJNI_GET_ARRAY_LENGTH, jsize (*)(JNIEnv*, jarray))(env, a);
}
static inline jobjectArray olfjni_NewObjectArray(JNIEnv* env, jsize len, jclass cls, jobject init) {
    return OLFJNI_FN(env, OLFJNI_NEW_OBJECT_ARRAY, jobjectArray (*)(JNIEnv*, jsize, jclass, jobject))(env, len, cls,
                                                                                                      init);
}
static inline jobject olfjni_GetObjectArrayElement(JNIEnv* env, jobjectArray a, jsize i) {
    return OLFJNI_FN(env, OLFJNI_GET_OBJECT_ARRAY_ELEMENT, jobject (*)(JNIEnv*, jobjectArray, jsize))(env, a, i);
}
static inline void olfjni_SetObjectArrayElement(JNIEnv* env, jobjectArray a, jsize i, jobject v) {
    OLFJNI_FN(env, OLFJNI_SET_OBJECT_ARRAY_ELEMENT, void (*)(JNIEnv*, jobjectArray, jsize, jobject))(env, a, i, v);
}
static inline jintArray olfjni_NewIntArray(JNIEnv* env, jsize len) {
    return OLFJNI_FN(env, OLFJNI_NEW_INT_ARRAY, jintArray (*)(JNIEnv*, jsize))(env, len);
}
static inline jdoubleArray olfjni_NewDoubleArray(JNIEnv* env, jsize len) {
    return OLFJNI_FN(env, OLFJNI_NEW_DOUBLE_ARRAY, jdoubleArray (*)(JNIEnv*, jsize))(env, len);
}
static inline void olfjni_GetBooleanArrayRegion(JNIEnv* env, jbooleanArray a, jsize start, jsize len, jboolean* buf) {
    OLFJNI_FN(env, OLFJNI_GET_BOOLEAN_ARRAY_REGION, void (*)(JNIEnv*, jbooleanArray, jsize, jsize, jboolean*))(
        env, a, start, len, buf);
}
static inline void olfjni_GetByteArrayRegion(JNIEnv* env, jbyteArray a, jsize start, jsize len, jbyte* buf) {
    OLFJNI_FN(env, OLFJNI_GET_BYTE_ARRAY_REGION, void (*)(JNIEnv*, jbyteArray, jsize, jsize, jbyte*))(env, a, start,
                                                                                                     len, buf);
}
static inline void olfjni_GetIntArrayRegion(JNIEnv* env, jintArray a, jsize start, jsize len, jint* buf) {
    OLFJNI_FN(env, OLFJNI_GET_INT_ARRAY_REGION, void (*)(JNIEnv*, jintArray, jsize, jsize, jint*))(env, a, start, len,
                                                                                                  buf);
}
static inline void olfjni_GetDoubleArrayRegion(JNIEnv* env, jdoubleArray a, jsize start, jsize len, jdouble* buf) {
    OLFJNI_FN(env, OLFJNI_GET_DOUBLE_ARRAY_REGION, void (*)(JNIEnv*, jdoubleArray, jsize, jsize, jdouble*))(
        env, a, start, len, buf);
}
static inline void olfjni_SetIntArrayRegion(JNIEnv* env, jintArray a, jsize start, jsize len, const jint* buf) {
    OLFJNI_FN(env, OLFJNI_SET_INT_ARRAY_REGION, void (*)(JNIEnv*, jintArray, jsize, jsize, const jint*))(env, a, start,
                                                                                                        len, buf);
}
static inline void olfjni_SetDoubleArrayRegion(JNIEnv* env, jdoubleArray a, jsize start, jsize len,
                                               const jdouble* buf) {
    OLFJNI_FN(env, OLFJNI_SET_DOUBLE_ARRAY_REGION, void (*)(JNIEnv*, jdoubleArray, jsize, jsize, const jdouble*))(
        env, a, start, len, buf);
}
static inline jboolean olfjni_ExceptionCheck(JNIEnv* env) {
    return OLFJNI_FN(env, OLFJNI_EXCEPTION_CHECK, jboolean (*)(JNIEnv*))(env);
}

#ifdef __cplusplus
}
#endif

#endif /* OLF_JNI_STUB_H */
