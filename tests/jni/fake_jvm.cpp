// TEST FIXTURE: a stand-in Java VM that drives the five exported JNI methods of
// br.unb.cic.tdp.base.GPUSortingSearch (tdp1375_b200/csrc/jni_bridge.cpp) the way the JVM
// would call them from GPUSortingSearch.java:30-45.  It implements the JNIEnv functions of
// tests/jni/jni.h over a small heap of Java arrays and records the pending exception, then
// prints one JSON line per call: the returned array (int[d][3] moves or byte[k][n] rows) or
// the RuntimeException message.
//
//   fake_jvm calls <file>   runs the calls listed in <file>, one per line:
//     init <totalSlots> <devices> <queueBytes> <dedupSize>
//     destroy
//     cancel <slot>
//     search <slot> <minRateBits> <maxMoves> <full> <initialEven> <n> <pi...> <spi...>
//     filter <skip> <n> <cycleLen> <cycle...> <tripleLen> <triple...>
#include <jni.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

extern "C" {
JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots(JNIEnv *, jclass, jint, jint, jlong, jint);
JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_destroySlots(JNIEnv *, jclass);
JNIEXPORT jobjectArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeq(
    JNIEnv *, jclass, jbyteArray, jbyteArray, jint, jfloat, jint, jboolean, jint);
JNIEXPORT void JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_cancelSort(JNIEnv *, jclass, jint);
JNIEXPORT jobjectArray JNICALL Java_br_unb_cic_tdp_base_GPUSortingSearch_filterPiPermutations(
    JNIEnv *, jclass, jbyteArray, jint, jbyteArray, jint, jint, jboolean);
}

namespace {

enum Kind { kClass, kIntArray, kByteArray, kObjectArray };

// Every Java object of this VM; the JNI handle is the object's address.
struct Obj : _jclass, _jintArray, _jbyteArray, _jobjectArray {
    Kind kind;
    std::string name;             // class name
    std::vector<jint> ints;       // int[]
    std::vector<jbyte> bytes;     // byte[]
    std::vector<Obj *> elements;  // Object[]
    int criticalPins = 0;
};

std::vector<std::unique_ptr<Obj>> gHeap;
std::string gPending;  // message of the pending RuntimeException ("" = none)
bool gHasPending = false;
int gLocalRefsDeleted = 0;

Obj *alloc(Kind k) {
    gHeap.push_back(std::make_unique<Obj>());
    gHeap.back()->kind = k;
    return gHeap.back().get();
}
Obj *obj(jobject o) { return static_cast<Obj *>(static_cast<_jclass *>(o)); }
Obj *obj(jarray a) {
    // every array handle the bridge passes back was produced by this VM from an Obj
    for (auto &h : gHeap) {
        if (static_cast<_jintArray *>(h.get()) == a || static_cast<_jbyteArray *>(h.get()) == a ||
            static_cast<_jobjectArray *>(h.get()) == a)
            return h.get();
    }
    std::fprintf(stderr, "unknown array handle\n");
    std::exit(3);
}

jboolean ExceptionCheck(JNIEnv *) { return gHasPending ? JNI_TRUE : JNI_FALSE; }
void ExceptionClear(JNIEnv *) {
    gHasPending = false;
    gPending.clear();
}
jclass FindClass(JNIEnv *, const char *name) {
    Obj *c = alloc(kClass);
    c->name = name;
    return static_cast<_jclass *>(c);
}
jint ThrowNew(JNIEnv *, jclass cls, const char *message) {
    if (obj(static_cast<jobject>(cls))->name != "java/lang/RuntimeException") std::exit(4);
    gHasPending = true;
    gPending = message ? message : "";
    return JNI_OK;
}
void DeleteLocalRef(JNIEnv *, jobject) { ++gLocalRefsDeleted; }
jsize GetArrayLength(JNIEnv *, jarray a) {
    Obj *o = obj(a);
    return (jsize)(o->kind == kIntArray ? o->ints.size() : o->kind == kByteArray ? o->bytes.size() : o->elements.size());
}
void *GetPrimitiveArrayCritical(JNIEnv *, jarray a, jboolean *isCopy) {
    Obj *o = obj(a);
    ++o->criticalPins;
    if (isCopy) *isCopy = JNI_FALSE;
    return o->kind == kIntArray ? (void *)o->ints.data() : (void *)o->bytes.data();
}
void ReleasePrimitiveArrayCritical(JNIEnv *, jarray a, void *, jint mode) {
    Obj *o = obj(a);
    if (mode != JNI_ABORT) std::exit(5);  // the bridge only reads its inputs
    --o->criticalPins;
}
jobjectArray NewObjectArray(JNIEnv *, jsize length, jclass, jobject) {
    Obj *o = alloc(kObjectArray);
    o->elements.assign((size_t)length, nullptr);
    return static_cast<_jobjectArray *>(o);
}
void SetObjectArrayElement(JNIEnv *, jobjectArray a, jsize index, jobject value) {
    Obj *o = obj(static_cast<jarray>(a));
    o->elements.at((size_t)index) = obj(static_cast<jarray>(static_cast<_jarray *>(static_cast<_jobject *>(value))));
}
jintArray NewIntArray(JNIEnv *, jsize length) {
    Obj *o = alloc(kIntArray);
    o->ints.assign((size_t)length, 0);
    return static_cast<_jintArray *>(o);
}
void SetIntArrayRegion(JNIEnv *, jintArray a, jsize start, jsize len, const jint *buf) {
    Obj *o = obj(static_cast<jarray>(a));
    for (jsize i = 0; i < len; ++i) o->ints.at((size_t)(start + i)) = buf[i];
}
jbyteArray NewByteArray(JNIEnv *, jsize length) {
    Obj *o = alloc(kByteArray);
    o->bytes.assign((size_t)length, 0);
    return static_cast<_jbyteArray *>(o);
}
void SetByteArrayRegion(JNIEnv *, jbyteArray a, jsize start, jsize len, const jbyte *buf) {
    Obj *o = obj(static_cast<jarray>(a));
    for (jsize i = 0; i < len; ++i) o->bytes.at((size_t)(start + i)) = buf[i];
}

const TdpTestJniFunctions kFunctions = {ExceptionCheck,   ExceptionClear,
                                        FindClass,        ThrowNew,
                                        DeleteLocalRef,   GetArrayLength,
                                        GetPrimitiveArrayCritical, ReleasePrimitiveArrayCritical,
                                        NewObjectArray,   SetObjectArrayElement,
                                        NewIntArray,      SetIntArrayRegion,
                                        NewByteArray,     SetByteArrayRegion};

jbyteArray byte_array(const std::vector<int> &v) {
    Obj *o = alloc(kByteArray);
    for (int x : v) o->bytes.push_back((jbyte)(uint8_t)x);  // Java bytes are signed: 200 is -56
    return static_cast<_jbyteArray *>(o);
}

std::string json_string(const std::string &s) {
    std::string out = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') out += '\\';
        out += c;
    }
    return out + "\"";
}

void report(const std::string &call, jobjectArray result) {
    std::printf("{\"call\": %s, ", json_string(call).c_str());
    if (gHasPending) {
        std::printf("\"exception\": %s, \"null_result\": %s}\n", json_string(gPending).c_str(),
                    result == nullptr ? "true" : "false");
        ExceptionClear(nullptr);
        return;
    }
    std::printf("\"exception\": null");
    if (result) {
        Obj *o = obj(static_cast<jarray>(result));
        std::printf(", \"rows\": [");
        for (size_t r = 0; r < o->elements.size(); ++r) {
            Obj *row = o->elements[r];
            std::printf("%s[", r ? ", " : "");
            const size_t len = row->kind == kIntArray ? row->ints.size() : row->bytes.size();
            for (size_t i = 0; i < len; ++i)
                std::printf("%s%d", i ? ", " : "",
                            row->kind == kIntArray ? row->ints[i] : (int)row->bytes[i]);
            std::printf("]");
        }
        std::printf("], \"row_kind\": \"%s\"",
                    o->elements.empty() ? "none" : (o->elements[0]->kind == kIntArray ? "int" : "byte"));
    }
    std::printf("}\n");
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 3 || std::strcmp(argv[1], "calls") != 0) {
        std::fprintf(stderr, "usage: fake_jvm calls <file>\n");
        return 2;
    }
    JNIEnv env{&kFunctions};
    jclass cls = FindClass(&env, "br/unb/cic/tdp/base/GPUSortingSearch");
    std::ifstream in(argv[2]);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        std::string op;
        if (!(ss >> op)) continue;
        if (op == "init") {
            long long slots, devices, queue, dedup;
            ss >> slots >> devices >> queue >> dedup;
            Java_br_unb_cic_tdp_base_GPUSortingSearch_initSlots(&env, cls, (jint)slots, (jint)devices, (jlong)queue,
                                                                (jint)dedup);
            report(line, nullptr);
        } else if (op == "destroy") {
            Java_br_unb_cic_tdp_base_GPUSortingSearch_destroySlots(&env, cls);
            report(line, nullptr);
        } else if (op == "cancel") {
            int slot;
            ss >> slot;
            Java_br_unb_cic_tdp_base_GPUSortingSearch_cancelSort(&env, cls, slot);
            report(line, nullptr);
        } else if (op == "search") {
            int slot, maxMoves, full, even, n, np, ns;
            unsigned rateBits;
            ss >> slot >> rateBits >> maxMoves >> full >> even >> n;
            std::vector<int> pi, spi;
            np = n;
            ns = n;
            if (n < 0) {  // a pi/spi length mismatch: |n| symbols of pi, |n|-1 of spi
                np = -n;
                ns = -n - 1;
            }
            for (int i = 0; i < np; ++i) {
                int v;
                ss >> v;
                pi.push_back(v);
            }
            for (int i = 0; i < ns; ++i) {
                int v;
                ss >> v;
                spi.push_back(v);
            }
            float rate;
            std::memcpy(&rate, &rateBits, 4);
            jobjectArray r = Java_br_unb_cic_tdp_base_GPUSortingSearch_searchForSortingSeq(
                &env, cls, byte_array(pi), byte_array(spi), even, rate, maxMoves, full ? JNI_TRUE : JNI_FALSE, slot);
            report(line, r);
        } else if (op == "filter") {
            int skip, n, cl, tl;
            ss >> skip >> n >> cl;
            std::vector<int> cycle(cl), triple;
            for (int &v : cycle) ss >> v;
            ss >> tl;
            triple.resize(tl);
            for (int &v : triple) ss >> v;
            jobjectArray r = Java_br_unb_cic_tdp_base_GPUSortingSearch_filterPiPermutations(
                &env, cls, byte_array(cycle), cl, byte_array(triple), tl, n, skip ? JNI_TRUE : JNI_FALSE);
            report(line, r);
        }
    }
    for (auto &h : gHeap)
        if (h->criticalPins != 0) {
            std::fprintf(stderr, "a critical array was not released\n");
            return 6;
        }
    return 0;
}
