// Host-side search slot: device buffers and launches for one stream on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tdp1375.h"
#include "engine.cuh"

namespace tdp {

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t e, const char *what)
        : std::runtime_error(std::string(what) + ": CUDA error " + cudaGetErrorName(e) + " (" +
                             cudaGetErrorString(e) + ")"),
          code(e) {}
};

void check(cudaError_t e, const char *what);

class SearchSlot {
public:
    SearchSlot(int device, int64_t queueBytesBudget, int dedupTableSize);
    ~SearchSlot();
    SearchSlot(const SearchSlot &) = delete;
    SearchSlot &operator=(const SearchSlot &) = delete;

    int device() const { return device_; }
    void cancel();
    void clearCancel();

    // Validates + uploads a batch; returns 0 or a TDP_ERR_* code (err holds the message).
    int stage(const tdp_instance *instances, int count, float minRate, std::string &err);
    // Runs the staged batch on the device and waits; 0 or TDP_ERR_DEVICE.
    int runStaged(std::string &err);
    // Copies the staged batch's results to the caller (in caller order).
    int fetch(tdp_result *results);
    int searchBatch(const tdp_instance *instances, int count, float minRate, tdp_result *results, std::string &err);

    tdp_stats stats() const;
    const tdp_engine_config &config() const { return cfg_; }
    // A new configuration invalidates a captured graph (its launch parameters change).
    void setConfig(const tdp_engine_config &c) {
        const int capacity = cfg_.task_capacity;
        cfg_ = c;
        cfg_.task_capacity = capacity;
        graphValid_ = false;
    }
    int stagedCount() const { return count_; }

    // Learned root ordering (n <= 32 instances of a batch).
    int setOrderModel(const uint16_t *w1, const float *b1, const uint16_t *w2, const float *b2, const uint16_t *w3,
                      const float *b3, const uint16_t *w4, const float *b4, std::string &err);
    bool hasOrderModel() const { return dW_[0] != nullptr; }
    // levels: 0 plain order, 1 learned root order, 2 learned root order and learned lists
    // at the first level below it
    void enableOrderModel(int levels) {
        orderEnabled_ = levels > 0;
        orderLevels_ = levels;
        graphValid_ = false;
    }

private:
    void ensureCapacity(int instances, int rules);
    void launchClass(int cls, int offset, int count);
    void wait();
    int computeRootOrder(int count, std::string &err);
    void prepareOrderBuffers(int count);

    int device_ = 0;
    int numSMs_ = 1;
    cudaStream_t stream_ = nullptr;
    cudaStream_t cancelStream_ = nullptr;
    cudaEvent_t evStart_ = nullptr, evStop_ = nullptr;
    int *dCancel_ = nullptr;
    int *hCancelValue_ = nullptr;
    std::atomic<bool> cancelRequested_{false};

    const uint32_t *triples_ = nullptr;
    void *dTable_ = nullptr;
    uint32_t tableEntries32_ = 0;
    uint32_t generation_ = 0;
    int lastLayout_ = -1;
    Mailbox *dMail_ = nullptr;
    int mailboxes_ = 0;
    uint32_t *dRing_ = nullptr;  // lap words then warp ids
    uint32_t ringSize_ = 0;
    EngineCtl *dCtl_ = nullptr;
    EngineCtl *hCtl_ = nullptr;  // two snapshots: one per size class

    InstanceIn *dIn_ = nullptr, *hIn_ = nullptr;
    InstanceOut *dOut_ = nullptr, *hOut_ = nullptr;
    uint32_t *dDone_ = nullptr;
    RuleTable *dRules_ = nullptr, *hRules_ = nullptr;
    int capInstances_ = 0, capRules_ = 0;

    std::vector<int> order_;
    int count_ = 0, countSmall_ = 0;

    tdp_engine_config cfg_{0, 64, 1, 0, 120.0, 2, 0, 0, 2, 1, 0};
    unsigned long long statsAccum_[kStatCount] = {};
    double kernelMs_ = 0.0;
    int deviceError_ = 0;
    int launches_ = 0;
    bool launched_[2] = {false, false};

    // ordering model: weights (bf16 [out x in]) and biases, inference scratch, root orders
    void *dW_[4] = {nullptr, nullptr, nullptr, nullptr};
    float *dB_[4] = {nullptr, nullptr, nullptr, nullptr};
    bool orderEnabled_ = false;
    int orderLevels_ = 0;
    // first-level lists: the states after the best kLevel1Ranks root children, scored by the
    // model, and each one's kLevel1List best children
    uint8_t *dL1Spi_ = nullptr, *dL1Pi_ = nullptr, *dL1N_ = nullptr;
    uint16_t *dOrder2_ = nullptr;
    int order2Cap_ = 0;
    void *dX_ = nullptr, *dH_[3] = {nullptr, nullptr, nullptr};
    float *dScores_ = nullptr;
    uint16_t *dOrder_ = nullptr;
    int orderCap_ = 0;
    int *dMlpErr_ = nullptr;
    bool orderedLaunch_ = false;

    // generation word (device) fed from pinned host memory, so a captured graph replays
    uint32_t *dGen_ = nullptr, *hGen_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graphExec_ = nullptr;
    bool graphValid_ = false;
    void enqueueRun(std::string &err, int &rc);
    void dropGraph();
};

}  // namespace tdp
