// extern "C" entry points: zeknox's C ABI (native/lib.h:21-51,
// native/merkle/merkle.h:30-62) over the B200 kernels, plus the stream-ordered
// extensions declared in include/zeknox.h.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <exception>
#include <string>
#include <vector>

#include "../../include/zeknox.h"
#include "fri.cuh"
#include "merkle.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

using namespace zk;

namespace {

thread_local int t_last_code = 0;
thread_local std::string t_last_msg;

}  // namespace

namespace zk {
void record_last_error(int code, const char *msg) {
    t_last_code = code;
    t_last_msg = msg ? msg : "";
}
}  // namespace zk

namespace {

RustError make_error(int code, const char *msg) {
    RustError r;
    r.code = code;
    r.message = (msg && *msg) ? strdup(msg) : nullptr;
    return r;
}

RustError ok() { return RustError{0, nullptr}; }

template <class F>
RustError guarded(F &&f) {
    try {
        f();
        return ok();
    } catch (const Error &e) {
        return make_error(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return make_error(-(int)cudaErrorMemoryAllocation, "host allocation failed");
    } catch (const std::exception &e) {
        return make_error(-(int)cudaErrorUnknown, e.what());
    }
}

// For the void entry points: remember the failure for zk_last_error().
template <class F>
void guarded_void(F &&f) {
    RustError r = guarded(f);
    if (r.code) {
        zk::record_last_error(r.code, r.message);
        fprintf(stderr, "zeknox-b200: %s\n", t_last_msg.c_str());
    }
    free(r.message);
}

// Rust binds device_id as i32 in places (wrappers/rust/src/lib.rs:51): only
// the low 32 bits are meaningful.
DeviceCtx &select(size_t device_id) {
    const int dev = (int)(uint32_t)device_id;
    ZK_CUDA(cudaSetDevice(dev));
    return device_ctx(dev);
}

void h2d(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes) ZK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
}
void d2h(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes) ZK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
}

uint64_t seed_now() {
    struct timespec ts;
    clock_gettime(CLOCK_REALTIME, &ts);
    return (uint64_t)ts.tv_sec * 1000000007ull ^ (uint64_t)ts.tv_nsec;
}

// The body of compute_batched_lde / zk_lde_async on device buffers.
void lde_device(DeviceCtx &ctx, uint64_t *d_out, const uint64_t *d_in, uint32_t lg_n, uint32_t rate_bits,
                uint64_t batches, bool inv, bool with_coset, cudaStream_t s) {
    const uint32_t lg = lg_n + rate_bits;
    require(lg <= (uint32_t)kMaxLg, "extended size 2^" + std::to_string(lg) + " out of range");
    const uint64_t N = 1ull << lg;
    NttJob j;
    j.src = d_in;
    j.src_stride = 1ull << lg_n;
    j.n_valid = 1ull << lg_n;
    j.dst = d_out;
    j.dst_stride = N;
    j.batches = batches;
    j.lg = lg;
    j.inverse = inv;
    if (with_coset) {
        const PowTable &c = coset_table(ctx, lg, GROUP_GENERATOR, false);
        (inv ? j.post_coset : j.pre_coset) = &c;
    }
    if (inv) j.scale = h_inv(1ull << lg);
    j.scratch_elems = ntt_scratch_elems(lg, batches);
    Scratch scr(j.scratch_elems * sizeof(uint64_t), s);
    j.scratch = scr.as<uint64_t>();
    ntt_run(j, s);
}

}  // namespace

namespace {
MerkleJob merkle_job(void *digests, void *cap, const void *leaves, uint64_t nd, uint64_t nc, uint64_t nl, uint64_t ls,
                     uint64_t ch, uint64_t ht) {
    MerkleJob j;
    j.digests = (uint64_t *)digests;
    j.cap = (uint64_t *)cap;
    j.leaves = (const uint64_t *)leaves;
    j.n_digests = nd;
    j.n_caps = nc;
    j.n_leaves = nl;
    j.leaf_size = ls;
    j.cap_height = ch;
    j.hash_type = ht;
    return j;
}
}  // namespace

// ------------------------------------------------------------------ devices

extern "C" RustError get_number_of_gpus(size_t *ngpus) {
    // zeknox counts devices of compute capability >= 7 (native/utils/all_gpus.cu:11-29).
    return guarded([&] {
        require(ngpus != nullptr, "null pointer");
        int n = device_count(), k = 0;
        for (int d = 0; d < n; d++) {
            int major = 0;
            if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d) == cudaSuccess && major >= 7) k++;
        }
        *ngpus = (size_t)k;
    });
}

extern "C" RustError list_devices_info(void) {
    return guarded([&] {
        int n = device_count();
        for (int d = 0; d < n; d++) {
            cudaDeviceProp p;
            ZK_CUDA(cudaGetDeviceProperties(&p, d));
            printf("GPU %d: %s, sm_%d%d, %d SMs, %.1f GiB, L2 %d MiB, %zu KiB smem/block (opt-in)\n", d, p.name,
                   p.major, p.minor, p.multiProcessorCount, p.totalGlobalMem / 1073741824.0, p.l2CacheSize >> 20,
                   p.sharedMemPerBlockOptin >> 10);
        }
    });
}

// ------------------------------------------------------------------ tables

extern "C" RustError init_twiddle_factors(size_t device_id, size_t lg_n) {
    return guarded([&] {
        DeviceCtx &c = select(device_id);
        require(lg_n >= 1 && lg_n <= (size_t)kMaxLg, "lg_n out of range");
        root_table(c, (unsigned)lg_n, false);
        root_table(c, (unsigned)lg_n, true);
        line_roots(c, false);
        line_roots(c, true);
    });
}

extern "C" RustError init_coset(size_t device_id, size_t lg_domain_size, const uint64_t coset_gen) {
    return guarded([&] {
        DeviceCtx &c = select(device_id);
        require(lg_domain_size <= (size_t)kMaxLg, "lg_domain_size out of range");
        coset_table(c, (unsigned)lg_domain_size, coset_gen % P_HOST, true);
    });
}

extern "C" void init_cuda_degree_and_generator(const uint32_t max_degree, const uint64_t group_generator) {
    guarded_void([&] {
        const int n = device_count();
        for (int d = 0; d < n; d++) {
            RustError r = init_coset((size_t)d, max_degree, group_generator);
            free(r.message);
            for (uint32_t k = 2; k <= max_degree && k <= (uint32_t)kMaxLg; k++) {
                r = init_twiddle_factors((size_t)d, k);
                free(r.message);
            }
        }
    });
}

extern "C" void init_cuda_degree(const uint32_t max_degree) { init_cuda_degree_and_generator(max_degree, GROUP_GENERATOR); }

extern "C" void init_cuda(void) { init_cuda_degree(24); }

// ---------------------------------------------------------------- NTT / LDE

// native/ntt/ntt.cu:253-309.  inverse: the inverse transform, then x coset^i
// (with_coset) and x 2^-lg.  forward: x coset^i (with_coset), then the
// transform.  Natural order in and out.
extern "C" RustError compute_batched_ntt(size_t device_id, void *inout, uint32_t lg_domain_size,
                                        NTT_Direction ntt_direction, NTT_Config cfg) {
    if (lg_domain_size == 0) return RustError{(int)cudaErrorInvalidValue, nullptr};
    return guarded([&] {
        DeviceCtx &ctx = select(device_id);
        const uint32_t lg = lg_domain_size;
        require(lg <= (uint32_t)kMaxLg, "lg_domain_size out of range");
        require(inout != nullptr || cfg.batches == 0, "null buffer");
        cudaStream_t s = ctx.stream;
        const uint64_t N = 1ull << lg, total = (uint64_t)cfg.batches << lg;
        const bool inv = ntt_direction == inverse;
        Scratch staging;
        uint64_t *d = (uint64_t *)inout;
        if (!cfg.are_inputs_on_device) {
            staging.alloc(total * sizeof(uint64_t), s);
            d = staging.as<uint64_t>();
            h2d(d, inout, total * sizeof(uint64_t), s);
        }
        NttJob j;
        j.src = d;
        j.dst = d;
        j.src_stride = j.dst_stride = N;
        j.n_valid = N;
        j.batches = cfg.batches;
        j.lg = lg;
        j.inverse = inv;
        if (cfg.with_coset) {
            const PowTable &c = coset_table(ctx, lg, GROUP_GENERATOR, false);
            (inv ? j.post_coset : j.pre_coset) = &c;
        }
        if (inv) j.scale = h_inv(N);
        j.scratch_elems = ntt_scratch_elems(lg, cfg.batches);
        Scratch scr(j.scratch_elems * sizeof(uint64_t), s);
        j.scratch = scr.as<uint64_t>();
        ntt_run(j, s);
        if (!cfg.are_inputs_on_device) d2h(inout, d, total * sizeof(uint64_t), s);
        ZK_CUDA(cudaStreamSynchronize(s));
    });
}

// native/ntt/ntt.cu:477-564: zero-extend each row from 2^lg_n to
// 2^(lg_n + rate_bits), then the transform above on the extended rows; salt
// rows (salt_size of them) are appended after the `batches` rows.
extern "C" RustError compute_batched_lde(size_t device_id, void *output, void *input, uint32_t lg_domain_size,
                                        NTT_Direction ntt_direction, NTT_Config cfg) {
    if (lg_domain_size == 0 || cfg.extension_rate_bits < 1)
        return make_error((int)cudaErrorInvalidValue, "invalid args");
    return guarded([&] {
        DeviceCtx &ctx = select(device_id);
        const uint32_t lg_n = lg_domain_size, rb = cfg.extension_rate_bits;
        require(lg_n + rb <= (uint32_t)kMaxLg, "extended size out of range");
        require((input && output) || cfg.batches + cfg.salt_size == 0, "null buffer");
        cudaStream_t s = ctx.stream;
        const uint64_t n = 1ull << lg_n, N = n << rb;
        const uint64_t in_total = (uint64_t)cfg.batches * n, out_total = (uint64_t)(cfg.batches + cfg.salt_size) * N;
        Scratch sin, sout;
        const uint64_t *d_in = (const uint64_t *)input;
        uint64_t *d_out = (uint64_t *)output;
        if (!cfg.are_inputs_on_device) {
            sin.alloc(in_total * sizeof(uint64_t), s);
            d_in = sin.as<uint64_t>();
        }
        if (!cfg.are_outputs_on_device) {
            sout.alloc(out_total * sizeof(uint64_t), s);
            d_out = sout.as<uint64_t>();
        }
        require(!(cfg.are_inputs_on_device && cfg.are_outputs_on_device && (const void *)d_in == (void *)d_out) ||
                    cfg.batches + cfg.salt_size == 0,
                "input and output must not alias");
        // Host buffers: polynomials go in groups, so that the copy of one group
        // overlaps the transform of another (copies on the context's copy
        // stream).  The groups' transforms alternate between two streams, so
        // that one group's tail overlaps the next group's start (four
        // separate 34-polynomial transforms cost 15 % more than one of 135).
        // Measured on 135 x 2^15 -> 2^18 from pinned memory: one stream and 4
        // groups 1.10 ms, two streams and 4 groups 0.98 ms, 8 groups 0.91 ms.
        const uint64_t B = cfg.batches;
        const uint64_t groups = (cfg.are_inputs_on_device && cfg.are_outputs_on_device) || B < 16 ? 1 : (B < 32 ? 4 : 8);
        const uint64_t gsz = (B + groups - 1) / std::max<uint64_t>(groups, 1);
        std::vector<cudaEvent_t> ev;
        auto event = [&](cudaStream_t st) {
            cudaEvent_t e;
            ZK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            ev.push_back(e);
            ZK_CUDA(cudaEventRecord(e, st));
            return e;
        };
        try {
            cudaStream_t cs = ctx.copy_stream;
            const cudaEvent_t allocated = event(s);
            ZK_CUDA(cudaStreamWaitEvent(cs, allocated, 0));  // after the allocations above
            const cudaStream_t lanes[2] = {s, groups > 1 ? ctx.lane_stream : s};
            if (groups > 1) ZK_CUDA(cudaStreamWaitEvent(lanes[1], allocated, 0));
            std::vector<cudaEvent_t> in_ready;
            for (uint64_t b0 = 0; b0 < B; b0 += gsz) {
                const uint64_t nb = std::min(gsz, B - b0);
                if (!cfg.are_inputs_on_device)
                    h2d(sin.as<uint64_t>() + b0 * n, (const uint64_t *)input + b0 * n, nb * n * sizeof(uint64_t), cs);
                in_ready.push_back(event(cs));
            }
            size_t gi = 0;
            for (uint64_t b0 = 0; b0 < B; b0 += gsz, gi++) {
                const uint64_t nb = std::min(gsz, B - b0);
                const cudaStream_t ls = lanes[gi & 1];
                ZK_CUDA(cudaStreamWaitEvent(ls, in_ready[gi], 0));
                lde_device(ctx, d_out + b0 * N, d_in + b0 * n, lg_n, rb, nb, ntt_direction == inverse, cfg.with_coset,
                           ls);
                if (!cfg.are_outputs_on_device) {
                    ZK_CUDA(cudaStreamWaitEvent(cs, event(ls), 0));
                    d2h((uint64_t *)output + b0 * N, d_out + b0 * N, nb * N * sizeof(uint64_t), cs);
                }
            }
            if (lanes[1] != s) ZK_CUDA(cudaStreamWaitEvent(s, event(lanes[1]), 0));  // join the second lane
            if (cfg.salt_size) {
                salt_run(d_out + B * N, (uint64_t)cfg.salt_size * N, seed_now(), s);
                if (!cfg.are_outputs_on_device) {
                    ZK_CUDA(cudaStreamWaitEvent(cs, event(s), 0));
                    d2h((uint64_t *)output + B * N, d_out + B * N, (uint64_t)cfg.salt_size * N * sizeof(uint64_t), cs);
                }
            }
            ZK_CUDA(cudaStreamWaitEvent(s, event(cs), 0));  // the stream-ordered frees come after the copies
            ZK_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamSynchronize(ctx.copy_stream);
            cudaStreamSynchronize(ctx.lane_stream);
            cudaStreamSynchronize(s);
            for (cudaEvent_t e : ev) cudaEventDestroy(e);
            throw;
        }
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    });
}

// native/ntt/ntt.cu:315-471.  One GPU here ("replicas only"): the input is a
// host buffer and the output a device buffer on GPU 0, as in zeknox.
extern "C" RustError compute_batched_lde_multi_gpu(void *output, void *input, uint32_t num_gpu,
                                                  NTT_Direction ntt_direction, NTT_Config cfg,
                                                  uint32_t lg_domain_size, size_t total_num_input_elements,
                                                  size_t total_num_output_elements) {
    (void)num_gpu;
    if (total_num_input_elements == 0 || lg_domain_size == 0 || cfg.extension_rate_bits < 1)
        return RustError{(int)cudaErrorInvalidValue, nullptr};
    if (total_num_input_elements < ((size_t)cfg.batches << lg_domain_size) ||
        total_num_output_elements < ((size_t)cfg.batches << (lg_domain_size + cfg.extension_rate_bits)))
        return make_error((int)cudaErrorInvalidValue, "buffer sizes smaller than the configured batch");
    NTT_Config c = cfg;
    c.are_inputs_on_device = false;
    c.are_outputs_on_device = true;
    c.salt_size = 0;
    return compute_batched_lde(0, output, input, lg_domain_size, ntt_direction, c);
}

// native/ntt/ntt.cu:182-226 / kernels.cu:94-135: out[rev(k)][b] = in[b][k].
extern "C" RustError compute_transpose_rev(size_t device_id, void *output, void *input, uint32_t lg_n,
                                          NTT_TransposeConfig cfg) {
    return guarded([&] {
        DeviceCtx &ctx = select(device_id);
        require(lg_n <= (uint32_t)kMaxLg, "lg_n out of range");
        require((input && output) || cfg.batches == 0, "null buffer");
        cudaStream_t s = ctx.stream;
        const uint64_t total = (uint64_t)cfg.batches << lg_n;
        Scratch sin, sout;
        const uint64_t *d_in = (const uint64_t *)input;
        uint64_t *d_out = (uint64_t *)output;
        if (!cfg.are_inputs_on_device) {
            sin.alloc(total * sizeof(uint64_t), s);
            h2d(sin.p, input, total * sizeof(uint64_t), s);
            d_in = sin.as<uint64_t>();
        }
        if (!cfg.are_outputs_on_device) {
            sout.alloc(total * sizeof(uint64_t), s);
            d_out = sout.as<uint64_t>();
        }
        require((const void *)d_in != (void *)d_out || total == 0, "transpose cannot run in place");
        transpose_rev_run(d_out, d_in, lg_n, cfg.batches, s);
        if (!cfg.are_outputs_on_device) d2h(output, d_out, total * sizeof(uint64_t), s);
        ZK_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" RustError compute_naive_transpose_rev(size_t device_id, void *output, void *input, uint32_t lg_n,
                                                NTT_TransposeConfig cfg) {
    return compute_transpose_rev(device_id, output, input, lg_n, cfg);
}

// ------------------------------------------------------------------- Merkle



// native/merkle/merkle.cu:246-280: enqueued on the legacy default stream of
// the current device, not synchronised (gpu_id is ignored, as in zeknox).
extern "C" void fill_digests_buf_linear_gpu_with_gpu_ptr(void *digests_buf_gpu_ptr, void *cap_buf_gpu_ptr,
                                                        void *leaves_buf_gpu_ptr, uint64_t digests_buf_size,
                                                        uint64_t cap_buf_size, uint64_t leaves_buf_size,
                                                        uint64_t leaf_size, uint64_t cap_height, uint64_t hash_type,
                                                        uint64_t gpu_id) {
    (void)gpu_id;
    guarded_void([&] {
        merkle_run(merkle_job(digests_buf_gpu_ptr, cap_buf_gpu_ptr, leaves_buf_gpu_ptr, digests_buf_size, cap_buf_size,
                              leaves_buf_size, leaf_size, cap_height, hash_type),
                   (cudaStream_t)0);
    });
}

// native/merkle/merkle.cu:462-499: buffers on GPU 0; one GPU here, and the
// call returns after the tree is complete.
extern "C" void fill_digests_buf_linear_multigpu_with_gpu_ptr(void *digests_buf_gpu_ptr, void *cap_buf_gpu_ptr,
                                                             void *leaves_buf_gpu_ptr, uint64_t digests_buf_size,
                                                             uint64_t cap_buf_size, uint64_t leaves_buf_size,
                                                             uint64_t leaf_size, uint64_t cap_height,
                                                             uint64_t hash_type) {
    guarded_void([&] {
        ZK_CUDA(cudaSetDevice(0));
        merkle_run(merkle_job(digests_buf_gpu_ptr, cap_buf_gpu_ptr, leaves_buf_gpu_ptr, digests_buf_size, cap_buf_size,
                              leaves_buf_size, leaf_size, cap_height, hash_type),
                   (cudaStream_t)0);
        ZK_CUDA(cudaStreamSynchronize((cudaStream_t)0));
    });
}

// native/merkle/merkle.cpp:126-161 takes host buffers; the same tree is built
// on the current GPU through staging buffers (no CPU fallback), synchronously.
extern "C" void fill_digests_buf_linear_cpu(void *digests_buf_ptr, void *cap_buf_ptr, const void *leaves_buf_ptr,
                                           uint64_t digests_buf_size, uint64_t cap_buf_size, uint64_t leaves_buf_size,
                                           uint64_t leaf_size, uint64_t cap_height, uint64_t hash_type) {
    guarded_void([&] {
        MerkleJob j = merkle_job(digests_buf_ptr, cap_buf_ptr, leaves_buf_ptr, digests_buf_size, cap_buf_size,
                                 leaves_buf_size, leaf_size, cap_height, hash_type);
        merkle_validate(j);
        DeviceCtx &ctx = select((size_t)current_device());
        cudaStream_t s = ctx.stream;
        const size_t lb = leaves_buf_size * leaf_size * sizeof(uint64_t);
        const size_t db = (j.n_caps == j.n_leaves ? 0 : digests_buf_size) * 4 * sizeof(uint64_t);
        const size_t cb = cap_buf_size * 4 * sizeof(uint64_t);
        Scratch dl(lb, s), dd(db, s), dc(cb, s);
        h2d(dl.p, leaves_buf_ptr, lb, s);
        // Digest words a hasher leaves untouched (Keccak on leaves shorter than
        // four words) keep the caller's values, as on zeknox's CPU path.
        h2d(dd.p, digests_buf_ptr, db, s);
        h2d(dc.p, cap_buf_ptr, cb, s);
        MerkleJob dj = j;
        dj.leaves = dl.as<uint64_t>();
        dj.digests = dd.as<uint64_t>();
        dj.cap = dc.as<uint64_t>();
        merkle_run(dj, s);
        d2h(digests_buf_ptr, dd.p, db, s);
        d2h(cap_buf_ptr, dc.p, cb, s);
        ZK_CUDA(cudaStreamSynchronize(s));
    });
}

// --------------------------------------------------------------- extensions

extern "C" RustError zk_last_error(void) {
    RustError r = t_last_code ? make_error(t_last_code, t_last_msg.c_str()) : ok();
    t_last_code = 0;
    t_last_msg.clear();
    return r;
}

extern "C" uint64_t zk_kernel_launches(void) { return launch_count(); }

extern "C" RustError zk_fill_field_async(void *d_out, uint64_t count, uint64_t seed, void *stream) {
    return guarded([&] {
        require(d_out != nullptr || count == 0, "null buffer");
        salt_run((uint64_t *)d_out, count, seed, (cudaStream_t)stream);
    });
}

extern "C" RustError zk_lde_async(void *d_output, const void *d_input, uint32_t lg_n, uint32_t rate_bits,
                                 uint32_t batches, uint32_t inv, uint32_t with_coset, void *stream) {
    return guarded([&] {
        require(lg_n >= 1 && rate_bits >= 1, "invalid args");
        DeviceCtx &ctx = select((size_t)current_device());
        require(d_output && d_input, "null buffer");
        lde_device(ctx, (uint64_t *)d_output, (const uint64_t *)d_input, lg_n, rate_bits, batches, inv != 0,
                   with_coset != 0, (cudaStream_t)stream);
    });
}

namespace {
// Forward coset LDE written in the leaf layout: leaves[rev(k)][b] = LDE_b[k].
// `coset` null: the installed coset generator (7 unless init_coset changed it).
void lde_leaves_device(DeviceCtx &ctx, uint64_t *d_leaves, const uint64_t *d_in, uint32_t lg_n, uint32_t rate_bits,
                       uint64_t batches, cudaStream_t s, const PowTable *coset = nullptr) {
    const uint32_t lg = lg_n + rate_bits;
    require(lg_n >= 1 && rate_bits >= 1 && lg <= (uint32_t)kMaxLg, "invalid args");
    NttJob j;
    j.src = d_in;
    j.src_stride = 1ull << lg_n;
    j.n_valid = 1ull << lg_n;
    j.dst = d_leaves;
    j.batches = batches;
    j.lg = lg;
    j.pre_coset = coset ? coset : &coset_table(ctx, lg, GROUP_GENERATOR, false);
    j.to_leaves = true;
    j.scratch_elems = ntt_leaves_scratch_elems(lg, batches);
    Scratch scr(j.scratch_elems * sizeof(uint64_t), s);
    j.scratch = scr.as<uint64_t>();
    ntt_run(j, s);
}
}  // namespace

extern "C" RustError zk_lde_leaves_async(void *d_leaves, const void *d_coeffs, uint32_t lg_n, uint32_t rate_bits,
                                        uint32_t batches, void *stream) {
    return guarded([&] {
        DeviceCtx &ctx = select((size_t)current_device());
        require(d_leaves && d_coeffs, "null buffer");
        lde_leaves_device(ctx, (uint64_t *)d_leaves, (const uint64_t *)d_coeffs, lg_n, rate_bits, batches,
                          (cudaStream_t)stream);
    });
}

extern "C" RustError zk_lde_leaves_coset_async(void *d_leaves, const void *d_coeffs, uint32_t lg_n,
                                              uint32_t rate_bits, uint32_t batches, uint64_t coset_gen,
                                              void *stream) {
    return guarded([&] {
        DeviceCtx &ctx = select((size_t)current_device());
        require(d_leaves && d_coeffs, "null buffer");
        require(coset_gen % P_HOST != 0, "coset generator must be non-zero");
        require(lg_n >= 1 && rate_bits >= 1 && lg_n + rate_bits <= (uint32_t)kMaxLg, "invalid args");
        const PowTable &t = shift_table(ctx, lg_n + rate_bits, coset_gen);
        lde_leaves_device(ctx, (uint64_t *)d_leaves, (const uint64_t *)d_coeffs, lg_n, rate_bits, batches,
                          (cudaStream_t)stream, &t);
    });
}

extern "C" RustError zk_fri_fold_async(void *d_out, const void *d_in, uint64_t n_in, uint32_t arity_bits,
                                      uint64_t beta0, uint64_t beta1, uint32_t in_interleaved, void *stream) {
    return guarded([&] {
        require(d_out && d_in, "null buffer");
        fri_fold_run((uint64_t *)d_out, (const uint64_t *)d_in, n_in, arity_bits, beta0, beta1, in_interleaved != 0,
                     (cudaStream_t)stream);
    });
}

extern "C" RustError zk_commit_async(const void *d_coeffs, uint32_t lg_n, uint32_t rate_bits, uint32_t batches,
                                    uint32_t cap_height, uint32_t hash_type, void *d_leaves, void *d_digests,
                                    void *d_cap, void *stream) {
    return guarded([&] {
        DeviceCtx &ctx = select((size_t)current_device());
        require(d_leaves && d_coeffs && d_cap, "null buffer");
        const uint64_t N = 1ull << (lg_n + rate_bits);
        const uint64_t nc = 1ull << cap_height;
        MerkleJob m = merkle_job(d_digests, d_cap, d_leaves, 2 * (N - nc), nc, N, batches, cap_height, hash_type);
        merkle_validate(m);  // before any work is queued
        lde_leaves_device(ctx, (uint64_t *)d_leaves, (const uint64_t *)d_coeffs, lg_n, rate_bits, batches,
                          (cudaStream_t)stream);
        merkle_run(m, (cudaStream_t)stream);
    });
}

extern "C" RustError zk_transpose_rev_async(void *d_output, const void *d_input, uint32_t lg_n, uint32_t batches,
                                           void *stream) {
    return guarded([&] {
        require(lg_n <= (uint32_t)kMaxLg, "lg_n out of range");
        require(d_output != d_input, "transpose cannot run in place");
        transpose_rev_run((uint64_t *)d_output, (const uint64_t *)d_input, lg_n, batches, (cudaStream_t)stream);
    });
}

extern "C" RustError zk_merkle_open_async(const void *d_leaves, const void *d_digests, uint64_t n_leaves,
                                         uint64_t leaf_size, uint64_t cap_height, const uint64_t *d_indices,
                                         uint64_t n_queries, void *d_out_leaves, void *d_out_siblings,
                                         void *stream) {
    return guarded([&] {
        merkle_open((const uint64_t *)d_leaves, (const uint64_t *)d_digests, n_leaves, leaf_size, cap_height,
                    d_indices, n_queries, (uint64_t *)d_out_leaves, (uint64_t *)d_out_siblings,
                    (cudaStream_t)stream);
    });
}

extern "C" RustError zk_merkle_async(void *d_digests, void *d_cap, const void *d_leaves, uint64_t n_digests,
                                    uint64_t n_caps, uint64_t n_leaves, uint64_t leaf_size, uint64_t cap_height,
                                    uint64_t hash_type, void *stream) {
    return guarded([&] {
        merkle_run(merkle_job(d_digests, d_cap, d_leaves, n_digests, n_caps, n_leaves, leaf_size, cap_height, hash_type),
                   (cudaStream_t)stream);
    });
}
