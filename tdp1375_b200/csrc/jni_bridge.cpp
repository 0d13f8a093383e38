// JNI bridge: the five native methods of br.unb.cic.tdp.base.GPUSortingSearch
// (GPUSortingSearch.java:30-45) over the C ABI of include/tdp1375.h.  Same symbol names,
// argument meaning and error behaviour as jni_sorter.cu:16-150: byte arrays are read
// unsigned and copied, results are fresh Java arrays owned by the caller, failures throw
// java.lang.RuntimeException with the native message and return null.
// Built only when a jni.h is available (tdp1375_b200/build.py).
#include <jni.h>

#include <cstdint>
#include <vector>

#include "../../include/tdp1375.h"

namespace {

void throw_runtime(JNIEnv *env, const char *message) {
    if (env->ExceptionCheck()) env->ExceptionClear();
    jclass cls = env->FindClass("java/lang/RuntimeException");
    if (cls) {
        env->ThrowNew(cls, message);
        env->DeleteLocalRef(cls);
    }
}

std::vector<uint8_t> copy_bytes(JNIEnv *env, jbyteArray array, jsize count) {
    std::vector<uint8_t> out((size_t)count);
    if (count > 0) {
        jbyte *p = static_cast<jbyte *>(env->GetPrimitiveArrayCritical(array, nullptr));
        if (p) {
            for (jsize i = 0; i < count; ++i) out[i] = static_cast<uint8_t>(p[i] & 0xFF);
            env->ReleasePrimitiveArrayCritical(array, p, JNI_ABORT);
        }
    }
    return out;
}

}  // namespace

extern "C" {

JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots(JNIEnv *env, jclass, jint totalSlots,
                                                                           jint devicesCount, jlong queueBytesBudget,
                                                                           jint dedupTableSize) {
    if (tdp_init_slots(totalSlots, devicesCount, queueBytesBudget, dedupTableSize) != 0)
        throw_runtime(env, tdp_last_error());
}

JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_destroySlots(JNIEnv *env, jclass) {
    if (tdp_destroy_slots() != 0) throw_runtime(env, tdp_last_error());
}

JNIEXPORT jobjectArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeq(
    JNIEnv *env, jclass, jbyteArray javaPi, jbyteArray javaSpi, jint initialEvenCycles, jfloat minRate,
    jint maxMoves, jboolean fullSorting, jint slot) {
    const jsize n = env->GetArrayLength(javaPi);
    if (env->GetArrayLength(javaSpi) != n) {
        throw_runtime(env, "performGpuSortingSearch: inconsistent input sizes");
        return nullptr;
    }
    const std::vector<uint8_t> pi = copy_bytes(env, javaPi, n);
    const std::vector<uint8_t> spi = copy_bytes(env, javaSpi, n);
    int32_t positions[3 * TDP_MAX_DEPTH];
    int32_t depth = 0;
    const int rc = tdp_search(slot, pi.data(), spi.data(), n, initialEvenCycles, minRate, maxMoves,
                              fullSorting ? 1 : 0, positions, &depth);
    if (rc != TDP_FOUND && rc != TDP_NOT_FOUND) {
        throw_runtime(env, tdp_last_error());
        return nullptr;
    }
    jclass intArrayClass = env->FindClass("[I");
    jobjectArray outer = env->NewObjectArray(depth, intArrayClass, nullptr);
    for (jsize d = 0; d < depth; ++d) {
        jint move[3] = {positions[3 * d], positions[3 * d + 1], positions[3 * d + 2]};
        jintArray inner = env->NewIntArray(3);
        env->SetIntArrayRegion(inner, 0, 3, move);
        env->SetObjectArrayElement(outer, d, inner);
        env->DeleteLocalRef(inner);
    }
    env->DeleteLocalRef(intArrayClass);
    return outer;
}

JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_cancelSort(JNIEnv *, jclass, jint slot) {
    tdp_cancel(slot);
}

JNIEXPORT jobjectArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_filterPiPermutations(
    JNIEnv *env, jclass, jbyteArray javaCycle, jint cycleLen, jbyteArray javaTriple, jint tripleLen, jint n,
    jboolean skip2MoveCheck) {
    const std::vector<uint8_t> cycle = copy_bytes(env, javaCycle, cycleLen);
    const std::vector<uint8_t> triple = copy_bytes(env, javaTriple, tripleLen);
    const int64_t maxRows = 1 << 20;  // MAX_OUTPUT of pi_filter.cu:16
    std::vector<uint8_t> rows((size_t)maxRows * (size_t)(n > 0 ? n : 1));
    const int64_t hits =
        tdp_pi_filter(cycle.data(), cycleLen, triple.data(), tripleLen, n, skip2MoveCheck ? 1 : 0, rows.data(), maxRows);
    if (hits < 0) {
        throw_runtime(env, tdp_last_error());
        return nullptr;
    }
    const jsize count = (jsize)(hits < maxRows ? hits : maxRows);
    jclass byteArrayClass = env->FindClass("[B");
    jobjectArray outer = env->NewObjectArray(count, byteArrayClass, nullptr);
    for (jsize r = 0; r < count; ++r) {
        jbyteArray inner = env->NewByteArray(n);
        env->SetByteArrayRegion(inner, 0, n, reinterpret_cast<const jbyte *>(rows.data() + (size_t)r * n));
        env->SetObjectArrayElement(outer, r, inner);
        env->DeleteLocalRef(inner);
    }
    env->DeleteLocalRef(byteArrayClass);
    return outer;
}

}  // extern "C"
