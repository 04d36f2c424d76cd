// abi.cu -- the exported C entry points (include/lib.h, include/merkle/merkle.h,
// include/zeknox_b200.h).
//
// Argument checks, host<->device staging and error codes follow zeknox
// native/lib.cu and native/ntt/ntt.cu; the computation is in ntt.cu/merkle.cu.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lib.h"
#include "../../include/zeknox_b200.h"
#include "batch.cuh"
#include "bounds.cuh"
#include "geom.h"
#include "gl64.cuh"
#include "multi_split.h"
#include "ntt_api.cuh"
#include "runtime.cuh"
#include "zk_constants.h"

bool zk_merkle_cpu(void *digests, void *caps, const void *leaves, uint64_t n_dig, uint64_t n_cap, uint64_t n_leaves,
                   uint64_t leaf_size, uint64_t cap_height, uint64_t hash_type, std::string &err);
// merkle_avx.cpp, compiled for AVX-512 and for AVX2 (call only on CPUs that have them)
extern "C" void zk_merkle_poseidon_avx512(uint64_t *dig, uint64_t *cap, const uint64_t *leaves, uint64_t n_dig,
                                          uint64_t n_cap, uint64_t n_leaves, uint64_t leaf_size, uint64_t cap_height);
extern "C" void zk_merkle_poseidon_avx2(uint64_t *dig, uint64_t *cap, const uint64_t *leaves, uint64_t n_dig,
                                        uint64_t n_cap, uint64_t n_leaves, uint64_t leaf_size, uint64_t cap_height);

namespace {

thread_local std::string g_last_error;

RustError ok() { return RustError{0, nullptr}; }

RustError fail(int code, const std::string &msg)
{
    RustError e;
    e.code = code;
    e.message = msg.empty() ? nullptr : strdup(msg.c_str());
    return e;
}

template <class F>
RustError guarded(F &&f)
{
    try {
        f();
        return ok();
    } catch (const zk::arg_failure &e) {
        return fail(e.code, e.what());
    } catch (const zk::cuda_failure &e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(-(int)cudaErrorMemoryAllocation, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(-(int)cudaErrorUnknown, e.what());
    }
}

void record_error(const char *fn, const std::string &msg)
{
    g_last_error = std::string(fn) + ": " + msg;
    fprintf(stderr, "zeknox: %s\n", g_last_error.c_str());
}

// Device copy of `elems` words at `p`: the pointer itself when on_device,
// otherwise a temporary filled from host memory (synchronously ordered on the
// device stream).
struct Staged {
    zk::DevBuf buf;
    uint64_t *dev = nullptr;
    Staged(zk::DeviceCtx &c, void *p, uint64_t elems, bool on_device, bool copy_in)
    {
        if (on_device) {
            dev = (uint64_t *)p;
        } else {
            buf.ctx = &c;
            buf.p = elems ? c.alloc(elems * 8) : nullptr;
            dev = buf.p;
            if (copy_in && elems) ZK_CUDA(cudaMemcpyAsync(dev, p, elems * 8, cudaMemcpyHostToDevice, c.stream));
        }
    }
};

// fn(g) for g < gpus, each on its own host thread so that every GPU's copies
// and kernels are issued at once (the reference issues all GPUs before it
// waits, native/ntt/ntt.cu:339-447, and runs one OpenMP thread per GPU,
// native/merkle/merkle.cu:392-451); the first failure is rethrown after all
// threads have finished.
template <class F>
void on_each_gpu(uint32_t gpus, F &&fn)
{
    if (gpus == 1) {
        fn(0u);
        return;
    }
    std::vector<std::exception_ptr> errs(gpus);
    std::vector<std::thread> threads;
    for (uint32_t g = 0; g < gpus; g++)
        threads.emplace_back([&, g] {
            try {
                fn(g);
            } catch (...) {
                errs[g] = std::current_exception();
            }
        });
    for (auto &t : threads) t.join();
    for (auto &e : errs)
        if (e) std::rethrow_exception(e);
}

}  // namespace

// ------------------------------------------------------------------ devices

extern "C" RustError get_number_of_gpus(size_t *ngpus)
{
    return guarded([&] {
        if (!ngpus) throw zk::arg_failure("null pointer");
        *ngpus = (size_t)zk::device_count();
    });
}

extern "C" RustError list_devices_info(void)
{
    return guarded([&] {
        int n = zk::device_count();
        for (int d = 0; d < n; d++) {
            cudaDeviceProp p;
            ZK_CUDA(cudaGetDeviceProperties(&p, d));
            printf("GPU %d: %s, sm_%d%d, %d SMs, %.1f GiB, L2 %d MiB, smem/block opt-in %zu KiB\n", d, p.name, p.major,
                   p.minor, p.multiProcessorCount, p.totalGlobalMem / 1073741824.0, p.l2CacheSize >> 20,
                   p.sharedMemPerBlockOptin >> 10);
            for (int q = 0; q < n; q++) {
                if (q == d) continue;
                int can = 0;
                ZK_CUDA(cudaDeviceCanAccessPeer(&can, d, q));
                printf("  peer %d -> %d: %s\n", d, q, can ? "yes" : "no");
            }
        }
    });
}

extern "C" bool cuda_available(void) { return zk::device_count() > 0; }

// ------------------------------------------------------------------- tables

extern "C" RustError init_twiddle_factors(size_t device_id, size_t lg_n)
{
    return guarded([&] {
        if (lg_n > 32) throw zk::arg_failure("lg_n above 32");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        c.twiddles((uint32_t)lg_n, false);
        c.twiddles((uint32_t)lg_n, true);
        c.sync();
    });
}

extern "C" RustError init_coset(size_t device_id, size_t lg_n, const uint64_t coset_gen)
{
    return guarded([&] {
        if (lg_n > 32) throw zk::arg_failure("lg_n above 32");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        c.set_coset((uint32_t)lg_n, coset_gen);
        c.sync();
    });
}

extern "C" void init_cuda_degree_and_generator(const uint32_t max_degree, const uint64_t group_generator)
{
    RustError e = guarded([&] {
        int n = zk::device_count();
        for (int d = 0; d < n; d++) {
            zk::DeviceCtx &c = zk::device(d);
            std::lock_guard<std::recursive_mutex> lk(c.mu);
            c.set_coset(max_degree, group_generator);
            for (uint32_t k = 1; k <= 12 && k <= max_degree; k++) {
                c.twiddles(k, false);
                c.twiddles(k, true);
            }
            c.sync();
        }
    });
    if (e.code) {
        record_error("init_cuda_degree_and_generator", e.message ? e.message : "error");
        free(e.message);
    }
}

extern "C" void init_cuda_degree(const uint32_t max_degree) { init_cuda_degree_and_generator(max_degree, ZK_GENERATOR); }

extern "C" void init_cuda(void) { init_cuda_degree(24); }

// --------------------------------------------------------------- transforms

extern "C" RustError compute_batched_ntt(size_t device_id, void *inout, uint32_t lg_domain_size,
                                         NTT_Direction ntt_direction, NTT_Config cfg)
{
    if (lg_domain_size == 0) return fail((int)cudaErrorInvalidValue, "lg_domain_size must be >= 1");
    return guarded([&] {
        if (lg_domain_size > 32) throw zk::arg_failure("lg_domain_size above 32");
        if (cfg.are_inputs_on_device != cfg.are_outputs_on_device)
            throw zk::arg_failure("in-place transform needs matching input/output placement");
        if (!inout && cfg.batches) throw zk::arg_failure("null buffer");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        const uint64_t total = (uint64_t)cfg.batches << lg_domain_size;
        Staged s(c, inout, total, cfg.are_inputs_on_device, true);
        zk::ntt_batch_device(c, s.dev, lg_domain_size, cfg.batches, ntt_direction == inverse, cfg.with_coset);
        if (!cfg.are_outputs_on_device && total)
            ZK_CUDA(cudaMemcpyAsync(inout, s.dev, total * 8, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

static void lde_on(zk::DeviceCtx &c, void *output, void *input, uint32_t lg_n, NTT_Direction dir, const NTT_Config &cfg)
{
    const uint64_t n = 1ULL << lg_n;
    const uint32_t rate = cfg.extension_rate_bits;
    const uint64_t N = n << rate;
    const uint64_t in_total = n * cfg.batches;
    const uint64_t out_total = N * ((uint64_t)cfg.batches + cfg.salt_size);
    Staged si(c, input, in_total, cfg.are_inputs_on_device, true);
    Staged so(c, output, out_total, cfg.are_outputs_on_device, false);
    zk::lde_batch_device(c, so.dev, si.dev, lg_n, rate, cfg.batches, dir == inverse, cfg.with_coset);
    if (cfg.salt_size) zk::salt_device(c, so.dev + N * cfg.batches, N * cfg.salt_size);
    if (!cfg.are_outputs_on_device && out_total)
        ZK_CUDA(cudaMemcpyAsync(output, so.dev, out_total * 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
}

extern "C" RustError compute_batched_lde(size_t device_id, void *output, void *input, uint32_t lg_domain_size,
                                         NTT_Direction ntt_direction, NTT_Config cfg)
{
    if (lg_domain_size == 0 || cfg.extension_rate_bits < 1) return fail((int)cudaErrorInvalidValue, "invalid args");
    return guarded([&] {
        if (cfg.extension_rate_bits > 32 || lg_domain_size > 32 - cfg.extension_rate_bits)
            throw zk::arg_failure("extended size above 2^32");
        if ((!input && cfg.batches) || (!output && (cfg.batches + cfg.salt_size))) throw zk::arg_failure("null buffer");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        lde_on(c, output, input, lg_domain_size, ntt_direction, cfg);
    });
}

extern "C" RustError compute_batched_lde_multi_gpu(void *output, void *input, uint32_t num_gpu,
                                                   NTT_Direction ntt_direction, NTT_Config cfg,
                                                   uint32_t lg_domain_size, size_t total_num_input_elements,
                                                   size_t total_num_output_elements)
{
    if (total_num_input_elements == 0 || lg_domain_size == 0 || cfg.extension_rate_bits < 1)
        return fail((int)cudaErrorInvalidValue, "invalid args");
    return guarded([&] {
        const uint32_t rate = cfg.extension_rate_bits;
        if (rate > 32 || lg_domain_size > 32 - rate) throw zk::arg_failure("extended size above 2^32");
        const uint64_t n = 1ULL << lg_domain_size, N = n << rate;
        if (total_num_input_elements < n * cfg.batches || total_num_output_elements < N * cfg.batches)
            throw zk::arg_failure("element counts smaller than batches x size");
        int ngpu = zk::device_count();
        uint32_t G = num_gpu == 0 ? 1 : num_gpu;
        if ((int)G > ngpu) throw zk::arg_failure("num_gpu exceeds the GPUs present");
        const zk::ColumnSplit sp = zk::split_columns(cfg.batches, G);
        // input in host memory (ntt.cu:360-364), output on GPU 0; every GPU
        // stages, transforms and copies its columns concurrently
        on_each_gpu(G, [&](uint32_t g) {
            if (!sp.take[g]) return;
            zk::DeviceCtx &c = zk::device(g);
            std::lock_guard<std::recursive_mutex> lk(c.mu);
            NTT_Config sub = cfg;
            sub.are_inputs_on_device = false;
            sub.are_outputs_on_device = true;
            sub.salt_size = 0;
            sub.batches = (uint32_t)sp.take[g];
            uint64_t *dst = (uint64_t *)output + sp.first[g] * N;
            uint64_t *src = (uint64_t *)input + sp.first[g] * n;
            if (g == 0) {
                lde_on(c, dst, src, lg_domain_size, ntt_direction, sub);
            } else {
                // computed on GPU g, then copied into GPU 0's output buffer
                zk::DevBuf tmp(c, sp.take[g] * N);
                lde_on(c, tmp.p, src, lg_domain_size, ntt_direction, sub);
                ZK_CUDA(cudaMemcpyPeerAsync(dst, 0, tmp.p, (int)g, sp.take[g] * N * 8, c.stream));
                c.sync();
            }
        });
    });
}

static RustError transpose_impl(size_t device_id, void *output, void *input, uint32_t lg_n, NTT_TransposeConfig cfg)
{
    return guarded([&] {
        if (lg_n > 32) throw zk::arg_failure("lg_n above 32");
        if (cfg.batches && (!input || !output)) throw zk::arg_failure("null buffer");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        const uint64_t total = (uint64_t)cfg.batches << lg_n;
        Staged si(c, input, total, cfg.are_inputs_on_device, true);
        Staged so(c, output, total, cfg.are_outputs_on_device, false);
        zk::transpose_rev_device(c, so.dev, si.dev, lg_n, cfg.batches);
        if (!cfg.are_outputs_on_device && total)
            ZK_CUDA(cudaMemcpyAsync(output, so.dev, total * 8, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

extern "C" RustError compute_transpose_rev(size_t device_id, void *output, void *input, uint32_t lg_n,
                                           NTT_TransposeConfig cfg)
{
    return transpose_impl(device_id, output, input, lg_n, cfg);
}

extern "C" RustError compute_naive_transpose_rev(size_t device_id, void *output, void *input, uint32_t lg_n,
                                                 NTT_TransposeConfig cfg)
{
    return transpose_impl(device_id, output, input, lg_n, cfg);
}

// The fused LDE with its leaf rows scattered over n_dst destination buffers
// (other GPUs' row shards, mapped for peer access): the LDE and the row
// exchange of a multi-GPU commit in one pass, the rows crossing NVLink as
// P2P stores straight from the row-writing kernel.
extern "C" RustError zeknox_lde_rows_scatter(size_t device_id, uint64_t *const *dst_ptrs, uint32_t n_dst,
                                             const uint64_t *coeffs, uint32_t lg_n, uint32_t rate_bits, uint32_t cols,
                                             uint32_t col_offset, uint32_t row_stride, uint64_t coset_gen, void *stream)
{
    return guarded([&] {
        if (lg_n == 0 || rate_bits == 0 || cols == 0) throw zk::arg_failure("lg_n, rate_bits and cols must be >= 1");
        if (rate_bits > 32 || lg_n > 32 - rate_bits) throw zk::arg_failure("extended size above 2^32");
        if (!dst_ptrs || !coeffs) throw zk::arg_failure("null buffer");
        const uint32_t lg_dst = zk::ilog2_exact(n_dst);
        if (lg_dst == ~0u || lg_dst > lg_n + rate_bits)
            throw zk::arg_failure("n_dst must be a power of two no larger than the row count");
        if ((uint64_t)col_offset + cols > row_stride) throw zk::arg_failure("columns beyond the destination rows");
        for (uint32_t d = 0; d < n_dst; d++)
            if (!dst_ptrs[d]) throw zk::arg_failure("null destination buffer");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        cudaStream_t keep = c.stream;
        if (stream) c.stream = (cudaStream_t)stream;
        try {
            zk::DevBuf tab(c, n_dst);
            ZK_CUDA(cudaMemcpyAsync(tab.p, dst_ptrs, n_dst * sizeof(uint64_t *), cudaMemcpyHostToDevice, c.stream));
            zk::RowScatter sc{(uint64_t *const *)tab.p, lg_n + rate_bits - lg_dst, col_offset, row_stride};
            zk::lde_rows_device(c, nullptr, coeffs, lg_n, rate_bits, cols, coset_gen ? coset_gen : ZK_GENERATOR, nullptr,
                                nullptr, &sc);
            // the pointer table is returned to the pool on the stream, after the kernels that read it
        } catch (...) {
            c.stream = keep;
            throw;
        }
        c.stream = keep;
        if (!stream) c.sync();
    });
}

// compute_transpose_rev of device buffers queued on the caller's stream
// (NULL: the device's stream, waited for), for pipelines that overlap it.
extern "C" RustError zeknox_transpose_rev(size_t device_id, uint64_t *output, const uint64_t *input, uint32_t lg_n,
                                          uint32_t cols, void *stream)
{
    return guarded([&] {
        if (lg_n > 32) throw zk::arg_failure("lg_n above 32");
        if (cols && (!input || !output)) throw zk::arg_failure("null buffer");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        cudaStream_t keep = c.stream;
        if (stream) c.stream = (cudaStream_t)stream;
        try {
            zk::transpose_rev_device(c, output, input, lg_n, cols);
        } catch (...) {
            c.stream = keep;
            throw;
        }
        c.stream = keep;
        if (!stream) c.sync();
    });
}

// ------------------------------------------------------------------- Merkle

extern "C" void fill_digests_buf_linear_gpu_with_gpu_ptr(void *digests_buf_gpu_ptr, void *cap_buf_gpu_ptr,
                                                         void *leaves_buf_gpu_ptr, u64 digests_buf_size,
                                                         u64 cap_buf_size, u64 leaves_buf_size, u64 leaf_size,
                                                         u64 cap_height, u64 hash_type, u64 gpu_id)
{
    (void)gpu_id;  // the reference ignores it too: pointers are on the current device
    std::string err;
    if (!zk::merkle_device((uint64_t *)digests_buf_gpu_ptr, (uint64_t *)cap_buf_gpu_ptr,
                           (const uint64_t *)leaves_buf_gpu_ptr, digests_buf_size, cap_buf_size, leaves_buf_size,
                           leaf_size, cap_height, hash_type, cudaStreamLegacy, err))
        record_error("fill_digests_buf_linear_gpu_with_gpu_ptr", err);
}

extern "C" void fill_digests_buf_linear_multigpu_with_gpu_ptr(void *digests_buf_gpu_ptr, void *cap_buf_gpu_ptr,
                                                              void *leaves_buf_gpu_ptr, u64 digests_buf_size,
                                                              u64 cap_buf_size, u64 leaves_buf_size, u64 leaf_size,
                                                              u64 cap_height, u64 hash_type)
{
    std::string err;
    if (!zk::merkle_geometry_ok(digests_buf_size, cap_buf_size, leaves_buf_size, cap_height, err)) {
        record_error("fill_digests_buf_linear_multigpu_with_gpu_ptr", err);
        return;
    }
    RustError e = guarded([&] {
        const uint64_t G = zk::merkle_gpu_count((uint64_t)zk::device_count(), cap_buf_size);
        const uint64_t L = leaves_buf_size / cap_buf_size, D = 2 * L - 2;
        const uint64_t caps_g = cap_buf_size / G;
        uint32_t hg = 0;
        while ((1ULL << hg) < caps_g) hg++;
        // GPU g builds subtrees [g * caps_g, (g + 1) * caps_g) from leaves
        // copied into its own memory (remote data lands locally before any
        // kernel reads it) and copies its digests and caps back to GPU 0; all
        // GPUs at once
        on_each_gpu((uint32_t)G, [&](uint32_t g) {
            zk::DeviceCtx &c = zk::device(g);
            std::lock_guard<std::recursive_mutex> lk(c.mu);
            const uint64_t leaves_g = caps_g * L, dig_g = caps_g * D;
            const uint64_t *src_leaves = (const uint64_t *)leaves_buf_gpu_ptr + g * leaves_g * leaf_size;
            uint64_t *dst_dig = (uint64_t *)digests_buf_gpu_ptr + g * dig_g * 4;
            uint64_t *dst_cap = (uint64_t *)cap_buf_gpu_ptr + g * caps_g * 4;
            if (G == 1) {
                std::string e2;
                if (!zk::merkle_device(dst_dig, dst_cap, src_leaves, digests_buf_size, cap_buf_size, leaves_buf_size,
                                       leaf_size, cap_height, hash_type, c.stream, e2))
                    throw zk::arg_failure(e2);
                c.sync();
                return;
            }
            zk::DevBuf lv(c, g ? leaves_g * leaf_size : 0), dg(c, g ? dig_g * 4 : 0), cp(c, g ? caps_g * 4 : 0);
            const uint64_t *use_leaves = src_leaves;
            uint64_t *use_dig = dst_dig, *use_cap = dst_cap;
            if (g) {
                ZK_CUDA(cudaMemcpyPeerAsync(lv.p, (int)g, src_leaves, 0, leaves_g * leaf_size * 8, c.stream));
                use_leaves = lv.p;
                use_dig = dg.p;
                use_cap = cp.p;
            }
            std::string e2;
            if (!zk::merkle_device(use_dig, use_cap, use_leaves, dig_g, caps_g, leaves_g, leaf_size, hg, hash_type,
                                   c.stream, e2))
                throw zk::arg_failure(e2);
            if (g) {
                ZK_CUDA(cudaMemcpyPeerAsync(dst_dig, 0, dg.p, (int)g, dig_g * 32, c.stream));
                ZK_CUDA(cudaMemcpyPeerAsync(dst_cap, 0, cp.p, (int)g, caps_g * 32, c.stream));
            }
            c.sync();
        });
    });
    if (e.code) {
        record_error("fill_digests_buf_linear_multigpu_with_gpu_ptr", e.message ? e.message : "error");
        free(e.message);
    }
}

extern "C" void fill_digests_buf_linear_cpu(void *digests_buf_ptr, void *cap_buf_ptr, const void *leaves_buf_ptr,
                                            u64 digests_buf_size, u64 cap_buf_size, u64 leaves_buf_size, u64 leaf_size,
                                            u64 cap_height, u64 hash_type)
{
    std::string err;
    if (!digests_buf_ptr || !cap_buf_ptr || !leaves_buf_ptr) {
        record_error("fill_digests_buf_linear_cpu", "null pointer");
        return;
    }
    if (!zk_merkle_cpu(digests_buf_ptr, cap_buf_ptr, leaves_buf_ptr, digests_buf_size, cap_buf_size, leaves_buf_size,
                       leaf_size, cap_height, hash_type, err))
        record_error("fill_digests_buf_linear_cpu", err);
}

// The reference's vector host builders (native/merkle/merkle.h:64-88,
// native/merkle/merkle_avx.cpp:189-276 and 451-538; exported there only from
// USE_AVX / USE_AVX512 builds): Poseidon only.  Here always exported; the
// forest is the one fill_digests_buf_linear_cpu builds (caps, digests and
// their layout), hashed W leaves per permutation on the vector units, or
// without them on a CPU that lacks the instruction set.  Unlike the reference:
// with caps == leaves the leaf hashes go to the caps (the reference's vector
// builders write them to the digests, which are empty then), and the AVX2
// builder hashes every leaf and node (the reference's steps by two, skipping
// odd ones).
static void merkle_cpu_vector(const char *who, bool avx512, void *digests_buf_ptr, void *cap_buf_ptr,
                              const void *leaves_buf_ptr, u64 digests_buf_size, u64 cap_buf_size, u64 leaves_buf_size,
                              u64 leaf_size, u64 cap_height, u64 hash_type)
{
    std::string err;
    if (!digests_buf_ptr || !cap_buf_ptr || !leaves_buf_ptr) {
        record_error(who, "null pointer");
        return;
    }
    if (!zk::merkle_geometry_check(digests_buf_size, cap_buf_size, leaves_buf_size, cap_height, err)) {
        record_error(who, err);
        return;
    }
    if (hash_type != 0) {  // HashPoseidon
        record_error(who, "only Poseidon (hash_type 0) has a vector host builder, got " + std::to_string(hash_type));
        return;
    }
    uint64_t *d = (uint64_t *)digests_buf_ptr, *c = (uint64_t *)cap_buf_ptr;
    const uint64_t *l = (const uint64_t *)leaves_buf_ptr;
    if (avx512 && __builtin_cpu_supports("avx512f"))
        zk_merkle_poseidon_avx512(d, c, l, digests_buf_size, cap_buf_size, leaves_buf_size, leaf_size, cap_height);
    else if (__builtin_cpu_supports("avx2"))
        zk_merkle_poseidon_avx2(d, c, l, digests_buf_size, cap_buf_size, leaves_buf_size, leaf_size, cap_height);
    else if (!zk_merkle_cpu(digests_buf_ptr, cap_buf_ptr, leaves_buf_ptr, digests_buf_size, cap_buf_size,
                            leaves_buf_size, leaf_size, cap_height, hash_type, err))
        record_error(who, err);
}

extern "C" void fill_digests_buf_linear_cpu_avx(void *digests_buf_ptr, void *cap_buf_ptr, const void *leaves_buf_ptr,
                                                u64 digests_buf_size, u64 cap_buf_size, u64 leaves_buf_size,
                                                u64 leaf_size, u64 cap_height, u64 hash_type)
{
    merkle_cpu_vector("fill_digests_buf_linear_cpu_avx", false, digests_buf_ptr, cap_buf_ptr, leaves_buf_ptr,
                      digests_buf_size, cap_buf_size, leaves_buf_size, leaf_size, cap_height, hash_type);
}

extern "C" void fill_digests_buf_linear_cpu_avx512(void *digests_buf_ptr, void *cap_buf_ptr, const void *leaves_buf_ptr,
                                                   u64 digests_buf_size, u64 cap_buf_size, u64 leaves_buf_size,
                                                   u64 leaf_size, u64 cap_height, u64 hash_type)
{
    merkle_cpu_vector("fill_digests_buf_linear_cpu_avx512", true, digests_buf_ptr, cap_buf_ptr, leaves_buf_ptr,
                      digests_buf_size, cap_buf_size, leaves_buf_size, leaf_size, cap_height, hash_type);
}

// -------------------------------------------------------------- extensions

extern "C" const char *zeknox_last_error(void) { return g_last_error.empty() ? nullptr : g_last_error.c_str(); }

extern "C" uint64_t zeknox_commit_scratch_words(const zk_commit_job *job)
{
    if (!job) return 0;
    return zk::commit_scratch_words(job->lg_n, job->rate_bits, job->cols, job->input_is_values != 0);
}

extern "C" RustError zeknox_commit(size_t device_id, const zk_commit_job *job, void *stream)
{
    return guarded([&] {
        if (!job) throw zk::arg_failure("null job");
        zk::check_job(*job);
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        cudaStream_t s = stream ? (cudaStream_t)stream : c.stream;
        const bool host_input = zk::is_host_pointer(job->input);
        const uint64_t words = zk::commit_scratch_words(job->lg_n, job->rate_bits, job->cols, job->input_is_values != 0,
                                                        host_input);
        zk::DevBuf scratch;
        if (words) {
            scratch.ctx = &c;
            cudaStream_t keep = c.stream;
            c.stream = s;  // allocate and free on the stream that uses it
            scratch.p = c.alloc(words * 8);
            c.stream = keep;
        }
        zk::commit_enqueue(c, *job, s, scratch.p, host_input);
        if (scratch.p) {
            (void)cudaFreeAsync(scratch.p, s);
            scratch.p = nullptr;
        }
        if (!stream) c.sync();
    });
}

extern "C" RustError zeknox_commit_batch(size_t device_id, const zk_commit_job *jobs, uint32_t njobs)
{
    return guarded([&] {
        if (njobs && !jobs) throw zk::arg_failure("null jobs");
        for (uint32_t i = 0; i < njobs; i++) zk::check_job(jobs[i]);
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        zk::commit_batch_graph(c, jobs, njobs);
        c.sync();
    });
}

extern "C" RustError zeknox_merkle_batch(size_t device_id, const zk_merkle_job *jobs, uint32_t njobs)
{
    return guarded([&] {
        if (njobs && !jobs) throw zk::arg_failure("null jobs");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        zk::merkle_batch_graph(c, jobs, njobs);
        c.sync();
    });
}

// ------------------------------------------------------------------ tuning

extern "C" RustError zeknox_tune_set(const char *name, uint32_t lg, uint64_t value)
{
    return guarded([&] {
        if (!name) throw zk::arg_failure("null knob name");
        zk::tune_set(name, lg, value);
    });
}

extern "C" uint64_t zeknox_tune_get(const char *name, uint32_t lg, uint64_t dflt)
{
    if (!name) return dflt;
    try {
        return zk::tune_get(name, lg, dflt);
    } catch (...) {
        return dflt;
    }
}

extern "C" RustError zeknox_tune_clear(void)
{
    return guarded([&] { zk::tune_clear(); });
}

// Table file: one knob per line, "<name> <lg or *> <value>"; '#' starts a comment.
extern "C" RustError zeknox_tune_load(const char *path)
{
    return guarded([&] {
        if (!path) throw zk::arg_failure("null path");
        zk::tune_load_file(path);
    });
}

// ------------------------------------------------------------- diagnostics

extern "C" uint64_t zeknox_launch_count(void) { return zk::launch_count(); }

extern "C" RustError zeknox_lde_rows(size_t device_id, uint64_t *rows, const uint64_t *coeffs, uint32_t lg_n,
                                     uint32_t rate_bits, uint32_t cols, uint64_t coset_gen, void *stream)
{
    return guarded([&] {
        if (lg_n == 0 || rate_bits == 0 || cols == 0) throw zk::arg_failure("lg_n, rate_bits and cols must be >= 1");
        if (rate_bits > 32 || lg_n > 32 - rate_bits) throw zk::arg_failure("extended size above 2^32");
        if (!rows || !coeffs) throw zk::arg_failure("null buffer");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        cudaStream_t keep = c.stream;
        if (stream) c.stream = (cudaStream_t)stream;
        try {
            zk::lde_rows_device(c, rows, coeffs, lg_n, rate_bits, cols, coset_gen ? coset_gen : ZK_GENERATOR, nullptr);
        } catch (...) {
            c.stream = keep;
            throw;
        }
        c.stream = keep;
        if (!stream) c.sync();
    });
}

// Out-of-range accesses the checked build's kernels skipped on this device
// since the last report: record = {count, first site, its index, its extent}.
extern "C" RustError zeknox_bounds_report(size_t device_id, uint64_t *record)
{
    if (!zk::BOUNDS_CHECKED) {
        if (record) record[0] = record[1] = record[2] = record[3] = 0;
        return fail((int)cudaErrorNotSupported, "range checks are compiled only into libzeknox_checked.so");
    }
    return guarded([&] {
        if (!record) throw zk::arg_failure("null record");
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        ZK_CUDA(cudaDeviceSynchronize());  // every queued kernel has recorded what it skipped
        uint64_t total[4] = {0, 0, 0, 0};
        for (auto take : {zk::oob_take_ntt, zk::oob_take_merkle, zk::oob_take_noalloc}) {
            uint64_t r[4];
            ZK_CUDA(take(r));
            if (r[0] && !total[0]) {
                total[1] = r[1];
                total[2] = r[2];
                total[3] = r[3];
            }
            total[0] += r[0];
        }
        for (int k = 0; k < 4; k++) record[k] = total[k];
    });
}

// Test hook for the bounded waits: the next `count` bulk-copy transposes on
// this device declare 16 bytes more than they copy, so one stage's wait runs
// out; the call that ran it returns -cudaErrorLaunchTimeout.
extern "C" RustError zeknox_inject_wait_timeout(size_t device_id, uint32_t count)
{
    return guarded([&] {
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        c.inject_wait_timeouts = count;
    });
}

// Register-resident Goldilocks multiply throughput: every thread runs 8
// independent chains x <- x * y of `iters` multiplies, with the lazily reduced
// product the permutations use (any 64-bit representative; IMAD selects the
// multiply-assisted reduction).  The faster of the two reductions is the
// ceiling of the permutations' multiply work.
template <bool IMAD>
__global__ void mul_rate_kernel(uint64_t *out, uint64_t seed, uint32_t iters)
{
    uint64_t x[8], y[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        x[i] = (seed + threadIdx.x * 8 + i) * 0x9E3779B97F4A7C15ULL % zk::GL_P;
        y[i] = (seed ^ (blockIdx.x * 131 + i)) * 0xBF58476D1CE4E5B9ULL % zk::GL_P;
    }
    for (uint32_t k = 0; k < iters; k++) {
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = zk::gl_mul_nc<IMAD>(x[i], y[i]);
    }
    uint64_t acc = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) acc ^= x[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

template <bool IMAD>
static double mul_rate_of(zk::DeviceCtx &c, uint64_t *out, int blocks, int threads, uint32_t iters)
{
    cudaEvent_t a, b;
    ZK_CUDA(cudaEventCreate(&a));
    ZK_CUDA(cudaEventCreate(&b));
    mul_rate_kernel<IMAD><<<blocks, threads, 0, c.stream>>>(out, 1, 64);  // warm-up
    ZK_CUDA(cudaEventRecord(a, c.stream));
    mul_rate_kernel<IMAD><<<blocks, threads, 0, c.stream>>>(out, 2, iters);
    ZK_CUDA(cudaEventRecord(b, c.stream));
    ZK_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    ZK_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return (double)blocks * threads * 8.0 * iters / (ms * 1e-3);
}

extern "C" double zeknox_measure_mul_rate(size_t device_id)
{
    double rate = -1;
    RustError e = guarded([&] {
        zk::DeviceCtx &c = zk::device(device_id);
        std::lock_guard<std::recursive_mutex> lk(c.mu);
        const int blocks = c.sm_count * 8, threads = 256;
        const uint32_t iters = 4096;
        zk::DevBuf out(c, (size_t)blocks * threads);
        const double alu = mul_rate_of<false>(c, out.p, blocks, threads, iters);
        const double imad = mul_rate_of<true>(c, out.p, blocks, threads, iters);
        rate = alu > imad ? alu : imad;
    });
    if (e.code) free(e.message);
    return rate;
}
