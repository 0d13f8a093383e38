// Host runtime of the search engine: per-slot device buffers, rule tables, launches.
#include "search_engine.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <map>
#include <vector>

#include "mlp.h"
#include "search_kernel.cuh"

namespace tdp {

namespace {

std::mutex gTripleMutex;
std::vector<uint32_t *> gTriples;  // per device

// Lexicographic (i<j<k) triples for every n in 3..63 at offset C(n,4) (the enumeration
// order of sorting_search.cu:750-758).
const uint32_t *device_triples(int device) {
    std::lock_guard<std::mutex> lock(gTripleMutex);
    if ((int)gTriples.size() <= device) gTriples.resize(device + 1, nullptr);
    if (gTriples[device]) return gTriples[device];
    const int total = combinations4(kMaxN + 1);
    std::vector<uint32_t> host((size_t)total, 0u);
    for (int n = 3; n <= kMaxN; ++n) {
        uint32_t *dst = host.data() + combinations4(n);
        int t = 0;
        for (int i = 0; i < n - 2; ++i)
            for (int j = i + 1; j < n - 1; ++j)
                for (int k = j + 1; k < n; ++k) dst[t++] = pack_triple(i, j, k);
    }
    uint32_t *d = nullptr;
    check(cudaMalloc(&d, host.size() * sizeof(uint32_t)), "cudaMalloc(triples)");
    check(cudaMemcpy(d, host.data(), host.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload triples");
    gTriples[device] = d;
    return d;
}

int count_even_host(const uint8_t *spi, int n) {
    uint64_t seen = 0;
    int count = 0;
    for (int s = 0; s < n; ++s) {
        if ((seen >> s) & 1ull) continue;
        int size = 0, cur = s;
        do {
            seen |= 1ull << cur;
            ++size;
            cur = spi[cur];
        } while (cur != s);
        count += size & 1;
    }
    return count;
}

bool is_permutation(const uint8_t *a, int n) {
    uint64_t seen = 0;
    for (int i = 0; i < n; ++i) {
        if (a[i] >= n) return false;
        if ((seen >> a[i]) & 1ull) return false;
        seen |= 1ull << a[i];
    }
    return true;
}

uint32_t round_pow2(uint64_t v) {
    uint64_t p = 8;
    while (p < v && p < (1ull << 31)) p <<= 1;
    return (uint32_t)p;
}

}  // namespace

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw CudaError(e, what);
}

SearchSlot::SearchSlot(int device, int64_t queueBytesBudget, int dedupTableSize) : device_(device) {
    check(cudaSetDevice(device), "cudaSetDevice");
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaStreamCreateWithFlags(&cancelStream_, cudaStreamNonBlocking), "cudaStreamCreate(cancel)");
    check(cudaMalloc(&dCancel_, sizeof(int)), "cudaMalloc(cancel)");
    check(cudaMemset(dCancel_, 0, sizeof(int)), "cudaMemset(cancel)");
    check(cudaHostAlloc(&hCancelValue_, sizeof(int), cudaHostAllocPortable), "cudaHostAlloc(cancel)");
    *hCancelValue_ = 1;
    check(cudaEventCreate(&evStart_), "cudaEventCreate");
    check(cudaEventCreate(&evStop_), "cudaEventCreate");
    triples_ = device_triples(device);
    check(cudaDeviceGetAttribute(&numSMs_, cudaDevAttrMultiProcessorCount, device), "SM count");

    tableEntries32_ = round_pow2((uint64_t)std::max(dedupTableSize, 1024));
    check(cudaMalloc(&dTable_, (size_t)tableEntries32_ * 32), "cudaMalloc(dedup table)");
    check(cudaMemset(dTable_, 0, (size_t)tableEntries32_ * 32), "cudaMemset(dedup table)");
    // One mailbox per warp of the largest grid this slot launches, and an idle-warp ring with
    // at least as many slots.  The queue budget of the reference (bytes for node queues)
    // bounds the mailbox area; the default budgets leave room for every resident warp.
    int maxBlocksPerSM = 0;
    check(cudaDeviceGetAttribute(&maxBlocksPerSM, cudaDevAttrMaxBlocksPerMultiprocessor, device), "blocks per SM");
    const int64_t warps = (int64_t)numSMs_ * std::min(maxBlocksPerSM, 8) * dev::kWarpsPerBlock;
    const int64_t byBudget = std::max<int64_t>(queueBytesBudget, 0) / (int64_t)sizeof(Mailbox);
    mailboxes_ = (int)std::max<int64_t>((int64_t)dev::kWarpsPerBlock * numSMs_,
                                        std::min<int64_t>(warps, std::max<int64_t>(byBudget, 1)));
    uint32_t ring = 1;
    while (ring < (uint32_t)mailboxes_) ring <<= 1;
    ringSize_ = ring;
    cfg_.task_capacity = mailboxes_;
    check(cudaMalloc(&dMail_, (size_t)mailboxes_ * sizeof(Mailbox)), "cudaMalloc(mailboxes)");
    check(cudaMalloc(&dRing_, (size_t)ringSize_ * 2 * sizeof(uint32_t)), "cudaMalloc(idle ring)");
    check(cudaMalloc(&dCtl_, sizeof(EngineCtl)), "cudaMalloc(ctl)");
    check(cudaMalloc(&dGen_, sizeof(uint32_t)), "cudaMalloc(generation)");
    check(cudaHostAlloc(&hGen_, 2 * sizeof(uint32_t), cudaHostAllocPortable), "cudaHostAlloc(generation)");
    check(cudaHostAlloc(&hCtl_, 2 * sizeof(EngineCtl), cudaHostAllocPortable), "cudaHostAlloc(ctl)");
    ensureCapacity(1, 1);
}

SearchSlot::~SearchSlot() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (cancelStream_) cudaStreamSynchronize(cancelStream_);
    cudaFree(dTable_);
    cudaFree(dMail_);
    cudaFree(dRing_);
    cudaFree(dCtl_);
    cudaFree(dIn_);
    cudaFree(dOut_);
    cudaFree(dRules_);
    cudaFree(dDone_);
    cudaFree(dCancel_);
    cudaFreeHost(hCtl_);
    cudaFreeHost(hIn_);
    cudaFreeHost(hOut_);
    cudaFreeHost(hRules_);
    cudaFreeHost(hCancelValue_);
    for (int l = 0; l < 4; ++l) {
        cudaFree(dW_[l]);
        cudaFree(dB_[l]);
    }
    cudaFree(dX_);
    for (int l = 0; l < 3; ++l) cudaFree(dH_[l]);
    cudaFree(dScores_);
    cudaFree(dOrder_);
    cudaFree(dOrder2_);
    cudaFree(dL1Spi_);
    cudaFree(dL1Pi_);
    cudaFree(dL1N_);
    cudaFree(dMlpErr_);
    dropGraph();
    cudaFree(dGen_);
    cudaFreeHost(hGen_);
    cudaEventDestroy(evStart_);
    cudaEventDestroy(evStop_);
    cudaStreamDestroy(stream_);
    cudaStreamDestroy(cancelStream_);
}

void SearchSlot::ensureCapacity(int instances, int rules) {
    if (instances > capInstances_) {
        const int cap = std::max(instances, capInstances_ * 2);
        cudaFree(dIn_);
        cudaFree(dOut_);
        cudaFree(dDone_);
        cudaFreeHost(hIn_);
        cudaFreeHost(hOut_);
        dIn_ = nullptr;
        dOut_ = nullptr;
        dDone_ = nullptr;
        hIn_ = nullptr;
        hOut_ = nullptr;
        check(cudaMalloc(&dIn_, (size_t)cap * sizeof(InstanceIn)), "cudaMalloc(instances)");
        check(cudaMalloc(&dOut_, (size_t)cap * sizeof(InstanceOut)), "cudaMalloc(results)");
        check(cudaMalloc(&dDone_, (size_t)((cap + 31) / 32) * sizeof(uint32_t)), "cudaMalloc(done bits)");
        check(cudaHostAlloc(&hIn_, (size_t)cap * sizeof(InstanceIn), cudaHostAllocPortable), "cudaHostAlloc(in)");
        check(cudaHostAlloc(&hOut_, (size_t)cap * sizeof(InstanceOut), cudaHostAllocPortable), "cudaHostAlloc(out)");
        capInstances_ = cap;
    }
    if (rules > capRules_) {
        const int cap = std::max(rules, std::max(64, capRules_ * 2));
        cudaFree(dRules_);
        cudaFreeHost(hRules_);
        dRules_ = nullptr;
        hRules_ = nullptr;
        check(cudaMalloc(&dRules_, (size_t)cap * sizeof(RuleTable)), "cudaMalloc(rules)");
        check(cudaHostAlloc(&hRules_, (size_t)cap * sizeof(RuleTable), cudaHostAllocPortable), "cudaHostAlloc(rules)");
        capRules_ = cap;
    }
}

void SearchSlot::clearCancel() {
    cancelRequested_.store(false);
    check(cudaSetDevice(device_), "cudaSetDevice");
    check(cudaStreamSynchronize(cancelStream_), "sync cancel stream");
    check(cudaMemsetAsync(dCancel_, 0, sizeof(int), stream_), "reset cancel flag");
}

void SearchSlot::cancel() {
    cancelRequested_.store(true);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device_);
    cudaMemcpyAsync(dCancel_, hCancelValue_, sizeof(int), cudaMemcpyHostToDevice, cancelStream_);
    if (prev >= 0 && prev != device_) cudaSetDevice(prev);
}

// Validates and stages instances (n <= 32 first, then n > 32) with their rule tables.
void SearchSlot::dropGraph() {
    if (graphExec_) cudaGraphExecDestroy(graphExec_);
    if (graph_) cudaGraphDestroy(graph_);
    graphExec_ = nullptr;
    graph_ = nullptr;
    graphValid_ = false;
}

int SearchSlot::stage(const tdp_instance *instances, int count, float minRate, std::string &err) {
    graphValid_ = false;
    order_.clear();
    order_.reserve(count);
    for (int pass = 0; pass < 2; ++pass)
        for (int i = 0; i < count; ++i)
            if ((instances[i].n > 32) == (pass == 1)) order_.push_back(i);
    countSmall_ = 0;
    for (int i = 0; i < count; ++i) countSmall_ += instances[i].n <= 32 ? 1 : 0;
    count_ = count;

    std::map<std::pair<uint64_t, uint64_t>, uint32_t> ruleIndex;
    std::vector<RuleTable> rules;
    ensureCapacity(std::max(count, 1), 1);
    uint32_t minRateBits;
    std::memcpy(&minRateBits, &minRate, 4);
    for (int slotIdx = 0; slotIdx < count; ++slotIdx) {
        const int src = order_[slotIdx];
        const tdp_instance &I = instances[src];
        const int n = I.n;
        if (n > kMaxN) {
            err = "performGpuSortingSearch: n exceeds MAX_N";
            return TDP_ERR_ARGUMENT;
        }
        if (I.max_depth <= 0 || I.max_depth > kMaxDepth) {
            err = "performGpuSortingSearch: invalid maximumDepth";
            return TDP_ERR_ARGUMENT;
        }
        if (!is_permutation(I.spi, n) || !is_permutation(I.pi, n)) {
            err = "tdp_search: spi and pi must be permutations of 0..n-1 (instance " + std::to_string(src) + ")";
            return TDP_ERR_ARGUMENT;
        }
        const std::pair<uint64_t, uint64_t> key(
            (uint64_t)n | ((uint64_t)I.max_depth << 8) | ((uint64_t)(I.full_sorting ? 1 : 0) << 16) |
                ((uint64_t)minRateBits << 32),
            (uint64_t)(uint32_t)I.initial_even_cycles);
        auto it = ruleIndex.find(key);
        uint32_t r;
        if (it == ruleIndex.end()) {
            RuleParams p{n, I.initial_even_cycles, I.max_depth, minRate, I.full_sorting ? 1 : 0};
            r = (uint32_t)rules.size();
            rules.push_back(build_rule_table(p, cfg_.tight_bound != 0));
            ruleIndex.emplace(key, r);
        } else {
            r = it->second;
        }
        InstanceIn &d = hIn_[slotIdx];
        std::memset(&d, 0, sizeof(d));
        std::memcpy(d.spi, I.spi, n);
        std::memcpy(d.pi, I.pi, n);
        d.n = (uint8_t)n;
        d.maxDepth = I.max_depth;
        d.even0 = (uint8_t)count_even_host(I.spi, n);
        d.rule = r;
    }
    ensureCapacity(std::max(count, 1), (int)std::max<size_t>(rules.size(), 1));
    if (!rules.empty()) std::memcpy(hRules_, rules.data(), rules.size() * sizeof(RuleTable));
    check(cudaSetDevice(device_), "cudaSetDevice");
    if (count > 0) {
        check(cudaMemcpyAsync(dIn_, hIn_, (size_t)count * sizeof(InstanceIn), cudaMemcpyHostToDevice, stream_),
              "upload instances");
        check(cudaMemcpyAsync(dRules_, hRules_, rules.size() * sizeof(RuleTable), cudaMemcpyHostToDevice, stream_),
              "upload rules");
    }
    return 0;
}

void SearchSlot::launchClass(int cls, int offset, int count) {
    if (count <= 0) return;
    // the generation word is copied from hGen_[cls], which runStaged set before this run
    check(cudaMemcpyAsync(dGen_, hGen_ + cls, sizeof(uint32_t), cudaMemcpyHostToDevice, stream_), "generation");
    check(cudaMemsetAsync(dCtl_, 0, sizeof(EngineCtl), stream_), "reset ctl");
    check(cudaMemsetAsync(dOut_ + offset, 0, (size_t)count * sizeof(InstanceOut), stream_), "reset results");
    check(cudaMemsetAsync(dDone_, 0, (size_t)((count + 31) / 32) * sizeof(uint32_t), stream_), "reset done bits");
    check(cudaMemsetAsync(dMail_, 0, (size_t)mailboxes_ * sizeof(Mailbox), stream_), "reset mailboxes");
    check(cudaMemsetAsync(dRing_, 0, (size_t)ringSize_ * sizeof(uint32_t), stream_), "reset idle ring");

    EngineParams P{};
    P.in = dIn_ + offset;
    P.out = dOut_ + offset;
    P.count = count;
    P.pollInterval = std::max(1, cfg_.poll_interval);
    P.rules = dRules_;
    P.triples = triples_;
    P.table = dTable_;
    P.tableMask = (cls == 0 ? tableEntries32_ : tableEntries32_ / 2) - 1u;
    P.generation = dGen_;
    P.doneBits = dDone_;
    P.mail = dMail_;
    P.ringSeq = dRing_;
    P.ringWid = dRing_ + ringSize_;
    P.ringMask = ringSize_ - 1u;
    P.ctl = dCtl_;
    P.cancel = dCancel_;
    P.timeLimitNs = (unsigned long long)(std::max(0.001, cfg_.time_limit_s) * 1e9);
    P.sparse = cfg_.sparse_enumeration;
    P.order = (cls == 0 && orderedLaunch_) ? dOrder_ : nullptr;
    P.orderStride = combinations3(32);
    P.order2 = (cls == 0 && orderedLaunch_ && orderLevels_ >= 2) ? dOrder2_ : nullptr;
    P.order2Ranks = kLevel1Ranks;
    P.order2List = kLevel1List;
    P.replace = cfg_.table_replacement;
    P.commute = cfg_.commute;
    P.probeLeaves = cfg_.probe_leaves;

    int blocksPerSM = 0;
    const int threads = dev::kWarpsPerBlock * 32;
    if (cls == 0) {
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocksPerSM, dev::search_engine_kernel<1>, threads, 0),
              "occupancy");
    } else {
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocksPerSM, dev::search_engine_kernel<2>, threads, 0),
              "occupancy");
    }
    if (cfg_.blocks_per_sm > 0) blocksPerSM = std::min(blocksPerSM, cfg_.blocks_per_sm);
    blocksPerSM = std::max(1, blocksPerSM);
    // every warp of the grid needs a mailbox
    const int grid = std::min(numSMs_ * blocksPerSM, mailboxes_ / dev::kWarpsPerBlock);
    P.maxInFlight = cfg_.warps_per_instance > 0
                        ? std::max(1, grid * dev::kWarpsPerBlock / cfg_.warps_per_instance)
                        : 0;
    if (cls == 0) {
        dev::search_engine_kernel<1><<<grid, threads, 0, stream_>>>(P);
    } else {
        dev::search_engine_kernel<2><<<grid, threads, 0, stream_>>>(P);
    }
    check(cudaGetLastError(), "launch search_engine_kernel");
    check(cudaMemcpyAsync(hCtl_ + cls, dCtl_, sizeof(EngineCtl), cudaMemcpyDeviceToHost, stream_), "read ctl");
    launched_[cls] = true;
    ++launches_;
}

// Waits for the slot stream while honouring the host cancel request (the device flag
// was already written by cancel()).
void SearchSlot::wait() {
    while (true) {
        const cudaError_t q = cudaStreamQuery(stream_);
        if (q == cudaSuccess) return;
        if (q != cudaErrorNotReady) check(q, "search kernel");
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

// Everything one batch run puts on the stream (root ordering, both size classes, control
// block read-back); captured once into a CUDA graph when use_cuda_graph is set.
void SearchSlot::enqueueRun(std::string &err, int &rc) {
    rc = 0;
    if (orderEnabled_ && hasOrderModel() && countSmall_ > 0) {
        rc = computeRootOrder(countSmall_, err);
        if (rc != 0) return;
        orderedLaunch_ = true;
    }
    launchClass(0, 0, countSmall_);
    launchClass(1, countSmall_, count_ - countSmall_);
}

int SearchSlot::runStaged(std::string &err) {
    check(cudaSetDevice(device_), "cudaSetDevice");
    deviceError_ = 0;
    launches_ = 0;
    std::fill(std::begin(statsAccum_), std::end(statsAccum_), 0ull);
    // Table generations: one per size class per run.  On wrap-around, or when the entry
    // layout changes, the table is cleared (outside any graph).
    for (int cls = 0; cls < 2; ++cls) {
        const int n = cls == 0 ? countSmall_ : count_ - countSmall_;
        if (n <= 0) continue;
        if (generation_ >= kMaxGeneration || cls != lastLayout_) {
            check(cudaMemsetAsync(dTable_, 0, (size_t)tableEntries32_ * 32, stream_), "clear dedup table");
            generation_ = 0;
            lastLayout_ = cls;
        }
        hGen_[cls] = ++generation_;
    }
    if (orderEnabled_ && hasOrderModel() && countSmall_ > 0) prepareOrderBuffers(countSmall_);
    check(cudaEventRecord(evStart_, stream_), "event");
    launched_[0] = launched_[1] = false;
    orderedLaunch_ = false;
    int rc = 0;
    if (cfg_.use_cuda_graph) {
        if (!graphValid_) {
            dropGraph();
            check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
            enqueueRun(err, rc);
            cudaGraph_t g = nullptr;
            const cudaError_t endErr = cudaStreamEndCapture(stream_, &g);
            if (rc != 0) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            check(endErr, "end capture");
            graph_ = g;
            check(cudaGraphInstantiate(&graphExec_, graph_, 0), "instantiate graph");
            graphValid_ = true;
        } else {
            launched_[0] = countSmall_ > 0;
            launched_[1] = count_ - countSmall_ > 0;
            launches_ = (launched_[0] ? 1 : 0) + (launched_[1] ? 1 : 0);
            orderedLaunch_ = orderEnabled_ && hasOrderModel() && countSmall_ > 0;
        }
        check(cudaGraphLaunch(graphExec_, stream_), "graph launch");
    } else {
        enqueueRun(err, rc);
        if (rc != 0) return rc;
    }
    check(cudaEventRecord(evStop_, stream_), "event");
    wait();
    for (int cls = 0; cls < 2; ++cls) {
        if (!launched_[cls]) continue;
        const EngineCtl &c = hCtl_[cls];
        for (int s = 0; s < kStatCount; ++s) statsAccum_[s] += c.stats[s];
        if (c.error != 0) deviceError_ = c.error;
    }
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, evStart_, evStop_), "elapsed");
    kernelMs_ = ms;
    if (orderedLaunch_) {
        int mlpErr = 0;
        check(cudaMemcpy(&mlpErr, dMlpErr_, sizeof(int), cudaMemcpyDeviceToHost), "read mlp error");
        if (mlpErr) {
            check(cudaMemset(dMlpErr_, 0, sizeof(int)), "reset mlp error");
            err = "ordering model: tensor-core pipeline wait timed out";
            return TDP_ERR_DEVICE;
        }
    }
    if (deviceError_ != 0) {
        err = deviceError_ == kErrDeadline ? "GPU sorting search exceeded its device time limit"
                                           : "GPU sorting search device error (spin limit)";
        if (!cancelRequested_.load()) return TDP_ERR_DEVICE;
    }
    return 0;
}

int SearchSlot::fetch(tdp_result *results) {
    check(cudaSetDevice(device_), "cudaSetDevice");
    if (count_ > 0) {
        check(cudaMemcpyAsync(hOut_, dOut_, (size_t)count_ * sizeof(InstanceOut), cudaMemcpyDeviceToHost, stream_),
              "read results");
        check(cudaStreamSynchronize(stream_), "sync results");
    }
    const bool cancelled = cancelRequested_.load();
    for (int slotIdx = 0; slotIdx < count_; ++slotIdx) {
        const InstanceOut &o = hOut_[slotIdx];
        tdp_result &r = results[order_[slotIdx]];
        std::memset(&r, 0, sizeof(r));
        r.nodes = o.nodes;
        r.children = o.children;
        if (o.state == kStateFound) {
            r.status = TDP_FOUND;
            r.depth = o.depth;
            for (int d = 0; d < o.depth && d < kMaxDepth; ++d) {
                r.positions[3 * d] = (int32_t)tri_i(o.moves[d]);
                r.positions[3 * d + 1] = (int32_t)tri_j(o.moves[d]);
                r.positions[3 * d + 2] = (int32_t)tri_k(o.moves[d]);
            }
        } else if (o.state == kStateNotFound) {
            r.status = TDP_NOT_FOUND;
        } else {
            r.status = cancelled ? TDP_CANCELLED : TDP_ERR_DEVICE;
        }
    }
    return 0;
}

int SearchSlot::searchBatch(const tdp_instance *instances, int count, float minRate, tdp_result *results,
                            std::string &err) {
    clearCancel();
    int rc = stage(instances, count, minRate, err);
    if (rc != 0) return rc;
    rc = runStaged(err);
    if (rc != 0) return rc;
    return fetch(results);
}

int SearchSlot::setOrderModel(const uint16_t *w1, const float *b1, const uint16_t *w2, const float *b2,
                              const uint16_t *w3, const float *b3, const uint16_t *w4, const float *b4,
                              std::string &err) {
    (void)err;
    check(cudaSetDevice(device_), "cudaSetDevice");
    const int rows[4] = {mlp::kHidden, mlp::kHidden, mlp::kHidden, mlp::kTriplesPadded};
    const int cols[4] = {mlp::kFeatures, mlp::kHidden, mlp::kHidden, mlp::kHidden};
    const int realRows[4] = {mlp::kHidden, mlp::kHidden, mlp::kHidden, mlp::kTriples};
    const uint16_t *w[4] = {w1, w2, w3, w4};
    const float *b[4] = {b1, b2, b3, b4};
    for (int l = 0; l < 4; ++l) {
        if (!dW_[l]) check(cudaMalloc(&dW_[l], (size_t)rows[l] * cols[l] * 2), "cudaMalloc(order weights)");
        if (!dB_[l]) check(cudaMalloc(&dB_[l], (size_t)rows[l] * sizeof(float)), "cudaMalloc(order bias)");
        check(cudaMemset(dW_[l], 0, (size_t)rows[l] * cols[l] * 2), "clear weights");
        check(cudaMemset(dB_[l], 0, (size_t)rows[l] * sizeof(float)), "clear bias");
        check(cudaMemcpy(dW_[l], w[l], (size_t)realRows[l] * cols[l] * 2, cudaMemcpyHostToDevice), "upload weights");
        check(cudaMemcpy(dB_[l], b[l], (size_t)realRows[l] * sizeof(float), cudaMemcpyHostToDevice), "upload bias");
    }
    if (!dMlpErr_) {
        check(cudaMalloc(&dMlpErr_, sizeof(int)), "cudaMalloc(mlp error)");
        check(cudaMemset(dMlpErr_, 0, sizeof(int)), "clear mlp error");
    }
    // one-time GEMM set-up (kernel attributes, tensor-map encoder) outside any capture
    if (mlp::prepare(err) != 0) return TDP_ERR_CUDA;
    graphValid_ = false;
    return 0;
}

// Scores every staged n <= 32 root with the MLP (tensor-core GEMMs on the slot stream, in
// chunks) and sorts its children by descending score into dOrder_.  With two levels it also
// builds the states after each root's kLevel1Ranks best children, scores them the same way
// and keeps each one's kLevel1List best children in dOrder2_.
constexpr int kOrderChunk = 8192;

// Buffers of the ordering pipeline; allocated before any graph capture.
void SearchSlot::prepareOrderBuffers(int count) {
    const int stride = combinations3(32);
    if (count > orderCap_) {
        cudaFree(dOrder_);
        dOrder_ = nullptr;
        check(cudaMalloc(&dOrder_, (size_t)count * stride * sizeof(uint16_t)), "cudaMalloc(order)");
        orderCap_ = count;
    }
    if (orderLevels_ >= 2 && count > order2Cap_) {
        cudaFree(dOrder2_);
        cudaFree(dL1Spi_);
        cudaFree(dL1Pi_);
        cudaFree(dL1N_);
        dOrder2_ = nullptr;
        dL1Spi_ = dL1Pi_ = dL1N_ = nullptr;
        const size_t rows = (size_t)count * kLevel1Ranks;
        check(cudaMalloc(&dOrder2_, rows * kLevel1List * sizeof(uint16_t)), "cudaMalloc(first-level order)");
        check(cudaMalloc(&dL1Spi_, rows * 64), "cudaMalloc(first-level states)");
        check(cudaMalloc(&dL1Pi_, rows * 64), "cudaMalloc(first-level states)");
        check(cudaMalloc(&dL1N_, rows), "cudaMalloc(first-level states)");
        order2Cap_ = count;
    }
    if (!dX_) {
        check(cudaMalloc(&dX_, (size_t)kOrderChunk * mlp::kFeatures * 2), "cudaMalloc(features)");
        for (int l = 0; l < 3; ++l)
            check(cudaMalloc(&dH_[l], (size_t)kOrderChunk * mlp::kHidden * 2), "cudaMalloc(hidden)");
        check(cudaMalloc(&dScores_, (size_t)kOrderChunk * mlp::kTriplesPadded * sizeof(float)), "cudaMalloc(scores)");
    }
}

int SearchSlot::computeRootOrder(int count, std::string &err) {
    constexpr int kChunk = kOrderChunk;
    const int stride = combinations3(32);
    const uint8_t *base = reinterpret_cast<const uint8_t *>(dIn_);
    // features -> 3 hidden layers -> scores for `rows` states; then rank them
    auto score = [&](const uint8_t *spi, const uint8_t *pi, const uint8_t *n, int rowStride, int nStride,
                     int rows) -> int {
        mlp::build_features(spi, pi, n, rowStride, nStride, rows, static_cast<__nv_bfloat16 *>(dX_), stream_);
        const void *in = dX_;
        int k = mlp::kFeatures;
        for (int l = 0; l < 3; ++l) {
            if (mlp::gemm_bf16(in, dW_[l], rows, mlp::kHidden, k, dB_[l], 1, dH_[l], 0, mlp::kHidden, dMlpErr_,
                               stream_, err) != 0)
                return TDP_ERR_CUDA;
            in = dH_[l];
            k = mlp::kHidden;
        }
        if (mlp::gemm_bf16(in, dW_[3], rows, mlp::kTriplesPadded, mlp::kHidden, dB_[3], 0, dScores_, 1,
                           mlp::kTriplesPadded, dMlpErr_, stream_, err) != 0)
            return TDP_ERR_CUDA;
        return 0;
    };
    for (int off = 0; off < count; off += kChunk) {
        const int rows = std::min(kChunk, count - off);
        const uint8_t *rec = base + (size_t)off * sizeof(InstanceIn);
        if (score(rec + offsetof(InstanceIn, spi), rec + offsetof(InstanceIn, pi), rec + offsetof(InstanceIn, n),
                  (int)sizeof(InstanceIn), (int)sizeof(InstanceIn), rows) != 0)
            return TDP_ERR_CUDA;
        mlp::order_by_score(dScores_, mlp::kTriplesPadded, rec + offsetof(InstanceIn, n), (int)sizeof(InstanceIn),
                            rows, dOrder_ + (size_t)off * stride, stride, stream_);
    }
    if (orderLevels_ >= 2) {
        mlp::level1_states(base + offsetof(InstanceIn, spi), base + offsetof(InstanceIn, pi),
                           base + offsetof(InstanceIn, n), (int)sizeof(InstanceIn), (int)sizeof(InstanceIn), count,
                           dOrder_, stride, kLevel1Ranks, dL1Spi_, dL1Pi_, dL1N_, stream_);
        const int states = count * kLevel1Ranks;
        for (int off = 0; off < states; off += kChunk) {
            const int rows = std::min(kChunk, states - off);
            if (score(dL1Spi_ + (size_t)off * 64, dL1Pi_ + (size_t)off * 64, dL1N_ + off, 64, 1, rows) != 0)
                return TDP_ERR_CUDA;
            mlp::top_k(dScores_, mlp::kTriplesPadded, dL1N_ + off, 1, rows, kLevel1List,
                       dOrder2_ + (size_t)off * kLevel1List, kLevel1List, stream_);
        }
    }
    check(cudaGetLastError(), "ordering model launch");
    return 0;
}

tdp_stats SearchSlot::stats() const {
    tdp_stats s{};
    s.nodes = statsAccum_[kStatNodes];
    s.children = statsAccum_[kStatChildren];
    s.dedup_probes = statsAccum_[kStatDedupProbes];
    s.dedup_pruned = statsAccum_[kStatDedupPruned];
    s.dedup_inserts = statsAccum_[kStatDedupInserts];
    s.dedup_full = statsAccum_[kStatDedupFull];
    s.donations = statsAccum_[kStatDonations];
    s.task_pops = statsAccum_[kStatTaskPops];
    s.busy_warp_cycles = statsAccum_[kStatBusyCycles];
    s.warp_cycles = statsAccum_[kStatWarpCycles];
    s.dedup_replaced = statsAccum_[kStatDedupReplaced];
    s.table_atomics = statsAccum_[kStatTableAtomics];
    s.commute_skips = statsAccum_[kStatCommuteSkips];
    s.kernel_ms = kernelMs_;
    s.error = deviceError_;
    s.launches = launches_;
    return s;
}

}  // namespace tdp
