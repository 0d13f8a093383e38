// Device data layout of the search engine (host and device share these structs).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tdp_math.cuh"

namespace tdp {

// Per-instance state machine (InstanceOut::state).
enum InstanceState : int {
    kStatePending = 0,
    kStateRunning = 1,
    kStateFound = 2,
    kStateNotFound = 3,
};

// One search instance as uploaded by the host (144 B).  spi/pi are the one-line arrays
// of the reference's JNI call (jni_sorter.cu:45-104, bytes read unsigned).
struct alignas(16) InstanceIn {
    uint8_t spi[64];
    uint8_t pi[64];
    uint8_t n;
    uint8_t maxDepth;
    uint8_t even0;  // odd-length cycles of spi, recounted on the host
    uint8_t flags;
    uint32_t rule;  // index into the RuleTable array
    uint32_t reserved[2];
};

// Result and live bookkeeping of one instance (96 B).
struct alignas(16) InstanceOut {
    int state;        // InstanceState
    int outstanding;  // tasks of this instance not yet finished
    int depth;        // solution length when found
    int reserved;
    unsigned long long nodes;     // expanded nodes
    unsigned long long children;  // children evaluated
    uint32_t moves[16];           // packed positions (pack_triple), depth entries
};

// A donated piece of work: the children [lo, hi) of one node at `depth` (in the index
// space of that node's enumeration mode; hi = 0xFFFF means all children), with the move
// path that reached it.  flags bit 0: the node has not been expanded yet (208 B).
struct alignas(16) Task {
    uint32_t inst;
    uint8_t depth;
    uint8_t even;
    uint8_t reserved0;
    uint8_t reserved1;
    uint16_t lo;
    uint16_t hi;
    uint32_t flags;                  // bit 0: unexpanded node; bits 8..15: first-level rank + 1
    uint32_t path[16];
    uint8_t spi[64];
    uint8_t pi[64];
};

enum EngineStat : int {
    kStatNodes = 0,
    kStatChildren,
    kStatDedupProbes,
    kStatDedupPruned,
    kStatDedupInserts,
    kStatDedupFull,
    kStatDonations,
    kStatTaskPops,
    kStatBusyCycles,  // SM cycles warps spent holding a task
    kStatWarpCycles,  // SM cycles of every warp from start to exit
    kStatDedupReplaced,  // inserts that overwrote a live entry of a full window
    kStatTableAtomics,   // transposition-table atomics issued (claims and depth updates)
    kStatCommuteSkips,   // children skipped by the partial-order reduction
    kStatCount
};

// Launch-wide control block, zeroed before every launch.  Fields that many warps touch
// live on separate 128-byte lines.
struct alignas(128) EngineCtl {
    unsigned ringHead;  // line 0: idle-warp ring, consumer side (donors)
    int pad0[31];
    unsigned ringTail;  // line 1: idle-warp ring, producer side (idle warps)
    int pad1[31];
    int nextInstance;  // line 2: instance admission / completion
    int doneCount;
    int pad2[30];
    int stop;  // line 3: launch stop + error
    int error;
    int pad3[30];
    unsigned long long stats[kStatCount];  // line 4
};

// Per-warp mailbox: a donor that dequeued this warp from the idle ring writes a Task here
// and then releases flag = 1; only the owning warp polls it.
struct alignas(256) Mailbox {
    Task task;
    uint32_t flag;
    uint32_t pad[11];
};

enum EngineError : int {
    kErrNone = 0,
    kErrSpinLimit = 1,
    kErrDeadline = 2,
};

// Learned order below the root: the best kLevel1Ranks root children each get a list of
// their kLevel1List best children, expanded first.
constexpr int kLevel1Ranks = 16;
constexpr int kLevel1List = 32;

constexpr uint32_t kTagWriting = 0xFFFFFFFFu;
constexpr uint32_t kMaxGeneration = 4094;  // generation 4095 would collide with kTagWriting
constexpr int kInstanceBits = 20;          // up to 1,048,576 instances per launch

// Transposition-table entry.  key = spi packed 5 bits/symbol, 12 per word (n <= 32) or
// 6 bits/symbol, 10 per word (n <= 63), in the low 60 bits of each word.
// tag = generation << 20 | instance.  meta = version << 13 | epoch << 5 | best depth.
// The version counts the entry's rewrites, and every key word carries the low 4 bits of the
// version that wrote it in its top 4 bits, so one read of the header and the key words tells
// whether the key belongs to the header: kernels may overwrite live entries of a full window,
// and a reader that meets a key word of another version treats the entry as unknown.
// The epoch is the write (or last useful read) time in units of 2^20 ns (8 bits, so ages up
// to ~268 ms compare correctly), used by the recency replacement policies.
template <int KW>
struct alignas(KW == 3 ? 32 : 64) DedupEntry {
    uint32_t tag;
    uint32_t meta;
    uint64_t key[KW];
};
constexpr uint32_t kDepthBits = 5;
constexpr uint32_t kDepthMask = (1u << kDepthBits) - 1u;
constexpr uint32_t kEpochShift = 5;
constexpr uint32_t kEpochMask = 255u << kEpochShift;
constexpr uint32_t kVersionShift = 13;
constexpr int kKeyCheckShift = 60;  // key word bits 60..63: version & 15 of the writer
constexpr uint64_t kKeyBits = (1ull << kKeyCheckShift) - 1ull;

struct EngineParams {
    const InstanceIn *in;
    InstanceOut *out;
    int count;
    int pollInterval;
    const RuleTable *rules;
    const uint32_t *triples;  // lexicographic (i,j,k) per n at offset combinations4(n)
    void *table;
    uint32_t tableMask;       // entries - 1 (entries of this launch's layout)
    const uint32_t *generation;  // device word: this launch's table generation (1..4094)
    uint32_t *doneBits;
    Mailbox *mail;            // one per warp of the grid
    uint32_t *ringSeq;        // idle-warp ring: per-slot lap word (zeroed per launch)
    uint32_t *ringWid;
    uint32_t ringMask;        // capacity - 1, capacity >= warps in the grid
    EngineCtl *ctl;
    const int *cancel;        // slot cancel flag (device)
    unsigned long long timeLimitNs;  // every warp stops (error kErrDeadline) after this long
    int sparse;                      // same-cycle pair enumeration allowed (n <= 32)
    const uint16_t *order;           // per-instance root child order (learned), or null
    int orderStride;
    const uint16_t *order2;          // per (instance, root rank < order2Ranks): best children of
                                     // that first-level node, order2List entries, or null
    int order2Ranks, order2List;
    int maxInFlight;                 // admitted-but-unfinished instance cap (0 = none)
    int replace;                     // full-window policy: 0 admit unrecorded, 1 deepest, 2 oldest,
                                     // 3 deepest then oldest (see dedup_admit_warp)
    int commute;                     // 1: partial-order reduction of commuting moves (por_skip)
    int probeLeaves;                 // 1: probe the table for children whose children are leaves
};

}  // namespace tdp
