// C ABI (include/tdp1375.h): slot table, argument checks, error mapping.
//
// Slot management follows slot_manager.cu:22-175 (slot s on device s % devicesCount, one
// non-blocking stream plus a cancel stream per slot, cancel = host flag + async write of
// the device flag) and the exception texts of sorting_search.cu:710-715, 841-846 and
// jni_sorter.cu.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/tdp1375.h"
#include "canonical.h"
#include "extension_filter.h"
#include "pi_filter.h"
#include "search_engine.h"

// The ABI structs have fixed sizes (the ctypes mirror in tdp1375_b200/native.py checks them too).
static_assert(sizeof(tdp_instance) == 136, "tdp_instance layout");
static_assert(sizeof(tdp_result) == 208, "tdp_result layout");
static_assert(sizeof(tdp_stats) == 120, "tdp_stats layout");
static_assert(sizeof(tdp_engine_config) == 48, "tdp_engine_config layout");

namespace {

thread_local std::string gLastError;
std::mutex gSlotsMutex;
std::vector<std::shared_ptr<tdp::SearchSlot>> gSlots;

int fail(int code, const std::string &msg) {
    gLastError = msg;
    return code;
}

std::shared_ptr<tdp::SearchSlot> get_slot(int slot) {
    std::lock_guard<std::mutex> lock(gSlotsMutex);
    if (slot < 0 || (size_t)slot >= gSlots.size() || !gSlots[slot]) return nullptr;
    return gSlots[slot];
}

int map_exception(const std::exception &e) {
    if (auto *ce = dynamic_cast<const tdp::CudaError *>(&e)) {
        if (ce->code == cudaErrorMemoryAllocation) return fail(TDP_ERR_OUT_OF_MEMORY, e.what());
        return fail(TDP_ERR_CUDA, e.what());
    }
    if (dynamic_cast<const std::bad_alloc *>(&e)) return fail(TDP_ERR_OUT_OF_MEMORY, "host allocation failed");
    return fail(TDP_ERR_CUDA, e.what());
}

}  // namespace

extern "C" {

const char *tdp_last_error(void) { return gLastError.c_str(); }

int tdp_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) return 0;
    return count;
}

int tdp_destroy_slots(void) {
    std::vector<std::shared_ptr<tdp::SearchSlot>> old;
    {
        std::lock_guard<std::mutex> lock(gSlotsMutex);
        old.swap(gSlots);
    }
    try {
        old.clear();
    } catch (const std::exception &e) {
        return map_exception(e);
    }
    return 0;
}

int tdp_init_slots(int total_slots, int devices_count, int64_t queue_bytes_budget, int dedup_table_size) {
    tdp_destroy_slots();
    if (total_slots <= 0 || devices_count <= 0) return fail(TDP_ERR_ARGUMENT, "initSlots: need at least one slot and one device");
    int available = tdp_device_count();
    if (available <= 0) return fail(TDP_ERR_CUDA, "initSlots: no CUDA device");
    if (devices_count > available) return fail(TDP_ERR_ARGUMENT, "initSlots: devicesCount exceeds the visible devices");
    int original = -1;
    cudaGetDevice(&original);
    std::vector<std::shared_ptr<tdp::SearchSlot>> slots;
    try {
        for (int s = 0; s < total_slots; ++s)
            slots.push_back(std::make_shared<tdp::SearchSlot>(s % devices_count, queue_bytes_budget, dedup_table_size));
    } catch (const std::exception &e) {
        if (original >= 0) cudaSetDevice(original);
        return map_exception(e);
    }
    if (original >= 0) cudaSetDevice(original);
    std::lock_guard<std::mutex> lock(gSlotsMutex);
    gSlots.swap(slots);
    return 0;
}

int tdp_cancel(int slot) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    s->cancel();
    return 0;
}

int tdp_search_batch(int slot, const tdp_instance *instances, int count, float min_rate, tdp_result *results) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (count < 0 || (count > 0 && (!instances || !results))) return fail(TDP_ERR_ARGUMENT, "tdp_search_batch: bad buffers");
    if (count > (1 << tdp::kInstanceBits)) return fail(TDP_ERR_ARGUMENT, "tdp_search_batch: at most 1048576 instances per call");
    try {
        std::string err;
        const int rc = s->searchBatch(instances, count, min_rate, results, err);
        if (rc != 0) return fail(rc, err);
        return 0;
    } catch (const std::exception &e) {
        return map_exception(e);
    }
}

int tdp_search(int slot, const uint8_t *pi, const uint8_t *spi, int n, int initial_even_cycles, float min_rate,
               int max_moves, int full_sorting, int32_t *out_positions, int32_t *out_depth) {
    if (out_depth) *out_depth = 0;
    if (n < 0 || (n > 0 && (!pi || !spi))) return fail(TDP_ERR_ARGUMENT, "performGpuSortingSearch: inconsistent input sizes");
    if (n > TDP_MAX_N) return fail(TDP_ERR_ARGUMENT, "performGpuSortingSearch: n exceeds MAX_N");
    if (max_moves <= 0 || max_moves > TDP_MAX_DEPTH)
        return fail(TDP_ERR_ARGUMENT, "performGpuSortingSearch: invalid maximumDepth");
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (n < 3) return TDP_NOT_FOUND;  // no triple: sorting_search.cu:718-719
    tdp_instance inst;
    std::memset(&inst, 0, sizeof(inst));
    inst.n = (uint8_t)n;
    inst.max_depth = (uint8_t)max_moves;
    inst.full_sorting = full_sorting ? 1 : 0;
    inst.initial_even_cycles = initial_even_cycles;
    std::memcpy(inst.pi, pi, n);
    std::memcpy(inst.spi, spi, n);
    tdp_result res;
    try {
        std::string err;
        const int rc = s->searchBatch(&inst, 1, min_rate, &res, err);
        if (rc != 0) return fail(rc, err);
    } catch (const std::exception &e) {
        return map_exception(e);
    }
    if (res.status == TDP_CANCELLED) return fail(TDP_CANCELLED, "GPU sorting search cancelled");
    if (res.status < 0) return fail(res.status, "GPU sorting search did not finish");
    if (res.status == TDP_FOUND) {
        if (out_depth) *out_depth = res.depth;
        if (out_positions) std::memcpy(out_positions, res.positions, sizeof(int32_t) * 3 * res.depth);
    }
    return res.status;
}

int tdp_batch_prepare(int slot, const tdp_instance *instances, int count, float min_rate) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (count < 0 || (count > 0 && !instances)) return fail(TDP_ERR_ARGUMENT, "tdp_batch_prepare: bad buffers");
    if (count > (1 << tdp::kInstanceBits)) return fail(TDP_ERR_ARGUMENT, "tdp_batch_prepare: at most 1048576 instances per call");
    try {
        std::string err;
        const int rc = s->stage(instances, count, min_rate, err);
        if (rc != 0) return fail(rc, err);
        return 0;
    } catch (const std::exception &e) {
        return map_exception(e);
    }
}

int tdp_batch_run(int slot) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    try {
        s->clearCancel();
        std::string err;
        const int rc = s->runStaged(err);
        if (rc != 0) return fail(rc, err);
        return 0;
    } catch (const std::exception &e) {
        return map_exception(e);
    }
}

int tdp_batch_results(int slot, tdp_result *results) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (!results && s->stagedCount() > 0) return fail(TDP_ERR_ARGUMENT, "tdp_batch_results: null buffer");
    try {
        return s->fetch(results);
    } catch (const std::exception &e) {
        return map_exception(e);
    }
}

int tdp_last_stats(int slot, tdp_stats *out) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (out) *out = s->stats();
    return 0;
}

int tdp_get_engine_config(int slot, tdp_engine_config *cfg) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (cfg) *cfg = s->config();
    return 0;
}

int tdp_set_engine_config(int slot, const tdp_engine_config *cfg) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (!cfg || cfg->poll_interval <= 0 || cfg->time_limit_s <= 0 || cfg->blocks_per_sm < 0 ||
        cfg->warps_per_instance < 0 || cfg->sparse_enumeration < 0 || cfg->sparse_enumeration > 2 ||
        cfg->table_replacement < 0 || cfg->table_replacement > 3 || cfg->commute < 0 || cfg->commute > 1 ||
        cfg->probe_leaves < 0 || cfg->probe_leaves > 1)
        return fail(TDP_ERR_ARGUMENT, "tdp_set_engine_config: invalid configuration");
    s->setConfig(*cfg);
    return 0;
}

double tdp_pi_filter_last_kernel_ms(void) { return tdp::gLastFilterKernelMs; }

int64_t tdp_pi_filter(const uint8_t *cycle, int cycle_len, const uint8_t *oriented_triple, int triple_len, int n,
                      int skip_2move_check, uint8_t *out, int64_t max_rows) {
    try {
        std::string err;
        const int64_t rc = tdp::pi_filter_run(cycle, cycle_len, oriented_triple, triple_len, n, skip_2move_check, out,
                                              max_rows, 600.0, err);
        if (rc >= 0) return rc;
        switch (rc) {
            case -1: return fail(TDP_ERR_ARGUMENT, err);
            case -4: return fail(TDP_ERR_OUT_OF_MEMORY, err);
            case -5: return fail(TDP_ERR_DEVICE, err);
            default: return fail(TDP_ERR_CUDA, err);
        }
    } catch (const std::exception &e) {
        return map_exception(e);
    }
}

}  // extern "C"

// ---------------------------------------------------------------- move-ordering MLP
#include "mlp.h"

namespace {

int *mlp_error_flag() {
    static std::mutex mu;
    static std::vector<int *> flags;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if ((int)flags.size() <= dev) flags.resize(dev + 1, nullptr);
    if (!flags[dev]) {
        int *p = nullptr;
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, sizeof(int));
        flags[dev] = p;
    }
    return flags[dev];
}

int launch_status(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(TDP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return 0;
}

}  // namespace

extern "C" {

int tdp_mlp_gemm(const void *a, const void *b, int m, int n, int k, const float *bias, int relu, void *out,
                 int out_fp32, int ldo, void *stream) {
    int *flag = mlp_error_flag();
    if (!flag) return fail(TDP_ERR_OUT_OF_MEMORY, "tdp_mlp_gemm: error flag allocation failed");
    std::string err;
    const int rc = tdp::mlp::gemm_bf16(a, b, m, n, k, bias, relu, out, out_fp32, ldo, flag,
                                       static_cast<cudaStream_t>(stream), err);
    if (rc != 0) return fail(rc == -1 ? TDP_ERR_ARGUMENT : TDP_ERR_CUDA, err);
    return 0;
}

int tdp_mlp_error(void) {
    int *flag = mlp_error_flag();
    if (!flag) return fail(TDP_ERR_OUT_OF_MEMORY, "tdp_mlp_error: error flag allocation failed");
    int host = 0;
    if (cudaMemcpy(&host, flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(TDP_ERR_CUDA, "tdp_mlp_error: read failed");
    if (host) cudaMemset(flag, 0, sizeof(int));
    return host;
}

int tdp_mlp_features(const uint8_t *spi, const uint8_t *pi, const uint8_t *n, int count, void *x, void *stream) {
    tdp::mlp::build_features(spi, pi, n, 64, 1, count, static_cast<__nv_bfloat16 *>(x), static_cast<cudaStream_t>(stream));
    return launch_status("tdp_mlp_features");
}

int tdp_mlp_softmax_xent(const float *logits, int ld, const uint8_t *n, const int32_t *target, int rows,
                         void *dlogits, float *loss, void *stream) {
    tdp::mlp::softmax_xent(logits, ld, n, target, rows, static_cast<__nv_bfloat16 *>(dlogits), loss,
                           static_cast<cudaStream_t>(stream));
    return launch_status("tdp_mlp_softmax_xent");
}

int tdp_mlp_transpose(const void *in, int rows, int cols, void *out, void *stream) {
    tdp::mlp::transpose_bf16(static_cast<const __nv_bfloat16 *>(in), rows, cols, static_cast<__nv_bfloat16 *>(out),
                             static_cast<cudaStream_t>(stream));
    return launch_status("tdp_mlp_transpose");
}

int tdp_mlp_relu_backward(void *grad, const void *act, int64_t count, void *stream) {
    tdp::mlp::relu_backward(static_cast<__nv_bfloat16 *>(grad), static_cast<const __nv_bfloat16 *>(act),
                            (size_t)count, static_cast<cudaStream_t>(stream));
    return launch_status("tdp_mlp_relu_backward");
}

int tdp_mlp_column_sums(const void *grad, int rows, int cols, float *out, void *stream) {
    tdp::mlp::column_sums(static_cast<const __nv_bfloat16 *>(grad), rows, cols, out, static_cast<cudaStream_t>(stream));
    return launch_status("tdp_mlp_column_sums");
}

int tdp_mlp_adam(float *master, void *weight, const float *grad, float *m, float *v, int64_t count, float lr,
                 float beta1, float beta2, float eps, int step, void *stream) {
    tdp::mlp::adam_step(master, static_cast<__nv_bfloat16 *>(weight), grad, m, v, (size_t)count, lr, beta1, beta2,
                        eps, step, static_cast<cudaStream_t>(stream));
    return launch_status("tdp_mlp_adam");
}

int tdp_mlp_order(const float *scores, int ld, const uint8_t *n, int count, uint16_t *order, int order_stride,
                  void *stream) {
    tdp::mlp::order_by_score(scores, ld, n, 1, count, order, order_stride, static_cast<cudaStream_t>(stream));
    return launch_status("tdp_mlp_order");
}

int tdp_set_order_model(int slot, const uint16_t *w1, const float *b1, const uint16_t *w2, const float *b2,
                        const uint16_t *w3, const float *b3, const uint16_t *w4, const float *b4) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (!w1 || !b1 || !w2 || !b2 || !w3 || !b3 || !w4 || !b4) return fail(TDP_ERR_ARGUMENT, "tdp_set_order_model: null array");
    try {
        std::string err;
        const int rc = s->setOrderModel(w1, b1, w2, b2, w3, b3, w4, b4, err);
        if (rc != 0) return fail(rc, err);
        return 0;
    } catch (const std::exception &e) {
        return map_exception(e);
    }
}

int tdp_enable_order_model(int slot, int enable) {
    auto s = get_slot(slot);
    if (!s) return fail(TDP_ERR_SLOT, "invalid slot");
    if (enable < 0 || enable > 2) return fail(TDP_ERR_ARGUMENT, "tdp_enable_order_model: levels must be 0, 1 or 2");
    if (enable && !s->hasOrderModel()) return fail(TDP_ERR_ARGUMENT, "tdp_enable_order_model: no model installed");
    s->enableOrderModel(enable);
    return 0;
}

}  // extern "C"

extern "C" int64_t tdp_pi_filter_noalloc(const uint8_t *cycle, int cycle_len, const uint8_t *oriented_triple,
                                         int triple_len, int n, int skip_2move_check, uint8_t *out_device,
                                         int64_t max_rows, void *stream) {
    std::string err;
    const int64_t rc = tdp::pi_filter_noalloc_run(cycle, cycle_len, oriented_triple, triple_len, n, skip_2move_check,
                                                  out_device, max_rows, static_cast<cudaStream_t>(stream), err);
    if (rc >= 0) return rc;
    return fail(rc == -1 ? TDP_ERR_ARGUMENT : TDP_ERR_CUDA, err);
}

extern "C" int tdp_extension_count(int n) { return (n < 3 || n > 60) ? 0 : tdp::extension_count(n); }

extern "C" int tdp_extension_filter_device(const uint8_t *spi, const uint8_t *pi, int n, int count, uint8_t *keep,
                                           void *stream) {
    std::string err;
    const int rc = tdp::extension_filter_device(spi, pi, n, count, keep, static_cast<cudaStream_t>(stream), err);
    if (rc != 0) return fail(rc == -1 ? TDP_ERR_ARGUMENT : TDP_ERR_CUDA, err);
    return 0;
}

extern "C" int64_t tdp_extension_filter(const uint8_t *spi, const uint8_t *pi, int n, int count, uint8_t *keep) {
    if (n < 3 || n > 60 || count < 0 || (count > 0 && (!spi || !pi || !keep)))
        return fail(TDP_ERR_ARGUMENT, "tdp_extension_filter: n must be in 3..60 with non-null buffers");
    if (count == 0) return 0;
    const size_t per = (size_t)tdp::extension_count(n), rows = (size_t)count * 64, total = (size_t)count * per;
    uint8_t *dSpi = nullptr, *dPi = nullptr, *dKeep = nullptr;
    auto release = [&] {
        cudaFree(dSpi);
        cudaFree(dPi);
        cudaFree(dKeep);
    };
    if (cudaMalloc(&dSpi, rows) != cudaSuccess || cudaMalloc(&dPi, rows) != cudaSuccess ||
        cudaMalloc(&dKeep, total) != cudaSuccess) {
        release();
        return fail(TDP_ERR_OUT_OF_MEMORY, "tdp_extension_filter: device allocation failed");
    }
    std::string err;
    int rc = 0;
    if (cudaMemcpy(dSpi, spi, rows, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dPi, pi, rows, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = -3, err = "tdp_extension_filter: upload failed";
    if (rc == 0) rc = tdp::extension_filter_device(dSpi, dPi, n, count, dKeep, nullptr, err);
    if (rc == 0 && cudaMemcpy(keep, dKeep, total, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = -3, err = "tdp_extension_filter: download failed";
    release();
    if (rc != 0) return fail(rc == -1 ? TDP_ERR_ARGUMENT : TDP_ERR_CUDA, err);
    int64_t hits = 0;
    for (size_t i = 0; i < total; ++i) hits += keep[i];
    return hits;
}

extern "C" int tdp_canonical_device(const uint8_t *spi, const uint8_t *n, int count, float *signature,
                                    int32_t *hash_code, int32_t *variant, void *stream) {
    std::string err;
    const int rc = tdp::canonical_device(spi, n, count, signature, hash_code, variant,
                                         static_cast<cudaStream_t>(stream), err);
    if (rc != 0) return fail(rc == -1 ? TDP_ERR_ARGUMENT : TDP_ERR_CUDA, err);
    return 0;
}

extern "C" int tdp_canonical(const uint8_t *spi, const uint8_t *n, int count, float *signature, int32_t *hash_code,
                             int32_t *variant) {
    if (count < 0 || (count > 0 && (!spi || !n || !signature || !hash_code || !variant)))
        return fail(TDP_ERR_ARGUMENT, "tdp_canonical: bad buffers");
    if (count == 0) return 0;
    std::string err;
    if (tdp::canonical_validate(spi, n, count, err) != 0) return fail(TDP_ERR_ARGUMENT, err);
    const size_t rows = (size_t)count * 64;
    uint8_t *dSpi = nullptr, *dN = nullptr;
    float *dSig = nullptr;
    int32_t *dHash = nullptr, *dVar = nullptr;
    auto release = [&] {
        cudaFree(dSpi);
        cudaFree(dN);
        cudaFree(dSig);
        cudaFree(dHash);
        cudaFree(dVar);
    };
    if (cudaMalloc(&dSpi, rows) != cudaSuccess || cudaMalloc(&dN, (size_t)count) != cudaSuccess ||
        cudaMalloc(&dSig, rows * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dHash, (size_t)count * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&dVar, (size_t)count * sizeof(int32_t)) != cudaSuccess) {
        release();
        return fail(TDP_ERR_OUT_OF_MEMORY, "tdp_canonical: device allocation failed");
    }
    int rc = 0;
    if (cudaMemcpy(dSpi, spi, rows, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dN, n, (size_t)count, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = -3, err = "tdp_canonical: upload failed";
    if (rc == 0) rc = tdp::canonical_device(dSpi, dN, count, dSig, dHash, dVar, nullptr, err);
    if (rc == 0 && (cudaMemcpy(signature, dSig, rows * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
                    cudaMemcpy(hash_code, dHash, (size_t)count * sizeof(int32_t), cudaMemcpyDeviceToHost) !=
                        cudaSuccess ||
                    cudaMemcpy(variant, dVar, (size_t)count * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = -3, err = "tdp_canonical: download failed";
    release();
    if (rc != 0) return fail(rc == -1 ? TDP_ERR_ARGUMENT : TDP_ERR_CUDA, err);
    return 0;
}
