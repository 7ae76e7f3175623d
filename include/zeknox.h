/*
 * zeknox-b200: the C ABI of zeknox's polynomial-commitment path, for one B200.
 *
 * Drop-in for the symbols zeknox exports from libzeknox (native/lib.h:21-51,
 * native/ntt/ntt.h:17-62, native/merkle/merkle.h:21-62): same names, the same
 * argument layout and meaning, the same RustError convention.  The Rust
 * (wrappers/rust/src/lib.rs:12-96) and Go (wrappers/go/lib/lib.go:7-212)
 * bindings link against libzeknox.so / libzeknox.a built from this tree
 * without change.  Extensions are marked as such.
 */
#ifndef ZEKNOX_B200_H
#define ZEKNOX_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ZK_VISIBLE __attribute__((visibility("default")))
#else
#define ZK_VISIBLE
#endif
#ifdef __cplusplus
#define ZK_EXTERN extern "C" ZK_VISIBLE
#define ZK_BOOL bool
#else
#define ZK_EXTERN ZK_VISIBLE
#define ZK_BOOL char /* C bindings (cgo) see one byte, as native/ntt/ntt.h:11-15 */
#endif

/* native/utils/rusterror.h:15-41: returned by value; code 0 = success, a
 * negative cudaError_t for CUDA failures, cudaErrorInvalidValue (1) for bad
 * arguments.  `message` is malloc'd (strdup) or NULL; the caller frees it. */
typedef struct RustError {
    int code;
    char *message;
} RustError;

/* native/ntt/ntt.h:17-41 */
typedef enum { NN, NR, RN, RR } NTT_InputOutputOrder;
typedef enum { forward, inverse } NTT_Direction;
typedef enum { standard, coset } NTT_Type;
typedef enum { GS, CT } NTT_Algorithm;

/* native/ntt/ntt.h:43-54 (24 bytes).  `order`, `ntt_type` and `is_multi_gpu`
 * are not read by the single-GPU path, as in zeknox. */
typedef struct {
    uint32_t batches;
    NTT_InputOutputOrder order;
    NTT_Type ntt_type;
    uint32_t extension_rate_bits;
    ZK_BOOL are_inputs_on_device;
    ZK_BOOL are_outputs_on_device;
    ZK_BOOL with_coset;
    ZK_BOOL is_multi_gpu;
    uint32_t salt_size;
} NTT_Config;

/* native/ntt/ntt.h:56-61 (8 bytes). */
typedef struct {
    uint32_t batches;
    ZK_BOOL are_inputs_on_device;
    ZK_BOOL are_outputs_on_device;
} NTT_TransposeConfig;

/* native/merkle/merkle.h:21-28 */
enum HashType { HashPoseidon = 0, HashKeccak = 1, HashPoseidonBN128 = 2, HashPoseidon2 = 3, HashMonolith = 4 };

#ifndef HASH_SIZE_U64
#define HASH_SIZE_U64 4
#endif

/* ---- device queries (native/lib.h:21-23; bodies native/lib.cu:36-70) ---- */
ZK_EXTERN RustError get_number_of_gpus(size_t *ngpus);
ZK_EXTERN RustError list_devices_info(void);

/* ---- table set-up (native/lib.h:25-31; native/lib.cu:115-175) ----
 * init_cuda() = init_cuda_degree(24); init_cuda_degree(d) =
 * init_cuda_degree_and_generator(d, 7): the coset table for 2^d points and the
 * twiddles for every size 2^2..2^d, on every GPU.  Tables are also built on
 * first use, so these calls are optional warm-ups here. */
ZK_EXTERN void init_cuda(void);
ZK_EXTERN void init_cuda_degree(const uint32_t max_degree);
ZK_EXTERN void init_cuda_degree_and_generator(const uint32_t max_degree, const uint64_t group_generator);
ZK_EXTERN RustError init_twiddle_factors(size_t device_id, size_t lg_n);
ZK_EXTERN RustError init_coset(size_t device_id, size_t lg_domain_size, const uint64_t coset_gen);

/* ---- NTT / LDE / transpose (native/lib.h:33-51; native/ntt/ntt.cu:182-564) ----
 * All synchronous.  Host buffers are staged through device memory owned by the
 * library.  Sizes: compute_batched_ntt works in place on batches * 2^lg
 * elements; compute_batched_lde reads batches * 2^lg_n and writes
 * (batches + salt_size) * 2^(lg_n + extension_rate_bits); transpose reads
 * batches * 2^lg_n and writes 2^lg_n rows of `batches` elements. */
ZK_EXTERN RustError compute_batched_ntt(size_t device_id, void *inout, uint32_t lg_domain_size,
                                        NTT_Direction ntt_direction, NTT_Config cfg);
ZK_EXTERN RustError compute_batched_lde(size_t device_id, void *output, void *input, uint32_t lg_domain_size,
                                        NTT_Direction ntt_direction, NTT_Config cfg);
ZK_EXTERN RustError compute_batched_lde_multi_gpu(void *output, void *input, uint32_t num_gpu,
                                                  NTT_Direction ntt_direction, NTT_Config cfg,
                                                  uint32_t lg_domain_size, size_t total_num_input_elements,
                                                  size_t total_num_output_elements);
ZK_EXTERN RustError compute_transpose_rev(size_t device_id, void *output, void *input, uint32_t lg_n,
                                          NTT_TransposeConfig cfg);
/* Declared by native/lib.h:50 but defined nowhere in zeknox; here an alias of
 * compute_transpose_rev. */
ZK_EXTERN RustError compute_naive_transpose_rev(size_t device_id, void *output, void *input, uint32_t lg_n,
                                                NTT_TransposeConfig cfg);

/* ---- Merkle (native/merkle/merkle.h:30-62; native/merkle/merkle.cu:246-280) ----
 * Linear digest layout: 2^cap_height subtrees, subtree s owns digests
 * [s*D, (s+1)*D) with D = digests_buf_size >> cap_height; leaf j of a subtree
 * sits at D - L + j (L = leaves per subtree); node i's children are 2(i+1) and
 * 2(i+1)+1; cap[s] = H(node 0, node 1).  Sizes count 4-element digests and
 * leaves.  The GPU variant takes device pointers, enqueues on the legacy
 * default stream and returns without synchronising (as zeknox does); gpu_id
 * is ignored and the current device is used.  Unsupported hash types return
 * without writing.  fill_digests_buf_linear_cpu takes host pointers and runs
 * the same kernels through staging buffers (synchronous). */
ZK_EXTERN void fill_digests_buf_linear_gpu_with_gpu_ptr(void *digests_buf_gpu_ptr, void *cap_buf_gpu_ptr,
                                                        void *leaves_buf_gpu_ptr, uint64_t digests_buf_size,
                                                        uint64_t cap_buf_size, uint64_t leaves_buf_size,
                                                        uint64_t leaf_size, uint64_t cap_height,
                                                        uint64_t hash_type, uint64_t gpu_id);
ZK_EXTERN void fill_digests_buf_linear_multigpu_with_gpu_ptr(void *digests_buf_gpu_ptr, void *cap_buf_gpu_ptr,
                                                             void *leaves_buf_gpu_ptr, uint64_t digests_buf_size,
                                                             uint64_t cap_buf_size, uint64_t leaves_buf_size,
                                                             uint64_t leaf_size, uint64_t cap_height,
                                                             uint64_t hash_type);
ZK_EXTERN void fill_digests_buf_linear_cpu(void *digests_buf_ptr, void *cap_buf_ptr, const void *leaves_buf_ptr,
                                           uint64_t digests_buf_size, uint64_t cap_buf_size,
                                           uint64_t leaves_buf_size, uint64_t leaf_size, uint64_t cap_height,
                                           uint64_t hash_type);

/* ================= extensions (no counterpart in zeknox) ================= */

/* Last error recorded by a void entry point on this thread (0 = none), e.g.
 * invalid Merkle sizes; cleared when read. */
ZK_EXTERN RustError zk_last_error(void);

/* Number of kernels this library has launched in this process. */
ZK_EXTERN uint64_t zk_kernel_launches(void);

/* count field elements uniform in [0, p) from seed, stream-ordered, into
 * d_out: element i is the first z(seed, i + j * count), j = 0, 1, ..., below p,
 * z(s, c) = SplitMix64's output function of s + (c + 1) * 0x9E3779B97F4A7C15
 * (the stream of the salt rows).  Synthetic inputs for tests and benchmarks. */
ZK_EXTERN RustError zk_fill_field_async(void *d_out, uint64_t count, uint64_t seed, void *stream);

/* Stream-ordered variants for callers that manage their own CUDA streams
 * (device pointers only, no synchronisation; `stream` is a cudaStream_t). */
ZK_EXTERN RustError zk_lde_async(void *d_output, const void *d_input, uint32_t lg_n, uint32_t rate_bits,
                                 uint32_t batches, uint32_t inv, uint32_t with_coset, void *stream);
ZK_EXTERN RustError zk_transpose_rev_async(void *d_output, const void *d_input, uint32_t lg_n, uint32_t batches,
                                           void *stream);
/* Forward coset LDE (generator 7, or the one init_coset installed) written
 * directly in the leaf layout of compute_transpose_rev: d_leaves[rev(k)][b] =
 * LDE_b[k], 2^(lg_n+rate_bits) rows of `batches` elements.  Equals
 * compute_batched_lde followed by compute_transpose_rev, without the
 * intermediate LDE matrix. */
ZK_EXTERN RustError zk_lde_leaves_async(void *d_leaves, const void *d_coeffs, uint32_t lg_n, uint32_t rate_bits,
                                        uint32_t batches, void *stream);
/* zk_lde_leaves_async on the coset coset_gen * <w_N> instead of the installed
 * one (the shifted cosets of FRI rounds: s_(i+1) = s_i^arity). */
ZK_EXTERN RustError zk_lde_leaves_coset_async(void *d_leaves, const void *d_coeffs, uint32_t lg_n,
                                              uint32_t rate_bits, uint32_t batches, uint64_t coset_gen,
                                              void *stream);
/* One FRI folding step over GF(p^2) = GF(p)[X]/(X^2 - 7) (no counterpart in
 * zeknox; the step of the Plonky2 prover that consumes its commitments):
 * d_out[j] = sum_(t < 2^arity_bits) beta^t * d_in[j * 2^arity_bits + t] for
 * j < n_in >> arity_bits, beta = beta0 + beta1 X.  d_out is in the split
 * layout (real parts, then the n_in >> arity_bits X parts); d_in is split
 * (2 rows of n_in) or, with in_interleaved, n_in (real, X) pairs (16-byte
 * aligned).  n_in a power of two, 1 <= arity_bits <= 6, canonical beta.  The
 * next round's leaves are zk_lde_leaves_coset_async(batches = 2) of d_out. */
ZK_EXTERN RustError zk_fri_fold_async(void *d_out, const void *d_in, uint64_t n_in, uint32_t arity_bits,
                                      uint64_t beta0, uint64_t beta1, uint32_t in_interleaved, void *stream);
/* One commit: zk_lde_leaves_async then the Merkle forest over those leaves
 * (digests 2*(N - 2^cap_height) x 4, cap 2^cap_height x 4, N = 2^(lg_n+rate_bits)). */
ZK_EXTERN RustError zk_commit_async(const void *d_coeffs, uint32_t lg_n, uint32_t rate_bits, uint32_t batches,
                                    uint32_t cap_height, uint32_t hash_type, void *d_leaves, void *d_digests,
                                    void *d_cap, void *stream);
/* Opening proofs on a resident forest (zeknox's linear layout, the output of
 * zk_merkle_async / fill_digests_buf_linear_gpu_with_gpu_ptr): for each of the
 * n_queries leaf indices in d_indices, its leaf row (leaf_size words, into
 * d_out_leaves) and the log2(n_leaves >> cap_height) sibling digests from the
 * leaf level up to the level below the cap (Plonky2's MerkleProof order), into
 * d_out_siblings (n_queries x depth x 4 words).  The path of leaf i ends at cap
 * entry i >> (log2(n_leaves) - cap_height).  Stream-ordered, device buffers;
 * a query index >= n_leaves gets all-ones words. */
ZK_EXTERN RustError zk_merkle_open_async(const void *d_leaves, const void *d_digests, uint64_t n_leaves,
                                         uint64_t leaf_size, uint64_t cap_height, const uint64_t *d_indices,
                                         uint64_t n_queries, void *d_out_leaves, void *d_out_siblings, void *stream);
ZK_EXTERN RustError zk_merkle_async(void *d_digests, void *d_cap, const void *d_leaves, uint64_t n_digests,
                                    uint64_t n_caps, uint64_t n_leaves, uint64_t leaf_size, uint64_t cap_height,
                                    uint64_t hash_type, void *stream);

/* Allocation-free coset LDE (no counterpart in zeknox).  Same arguments and
 * result as zk_lde_async (device buffers, stream-ordered, the installed coset
 * generator: 7 unless init_coset set another) for callers that cannot call
 * cudaMalloc where they run it: provers confined to a pre-reserved memory
 * budget or their own arena (the regular entry points grow the CUDA memory
 * pool), and hot paths where allocation calls are forbidden because they can
 * synchronise the device.  Its NTT intermediate and tables live in one static
 * device array (32 MiB + 96 KiB per GPU, held until exit), so: lg_n +
 * rate_bits must be <= 22 (else code cudaErrorMemoryAllocation = 2, NULL
 * message); calls that overlap on the GPU race on the shared array; the first
 * call on a device resolves the array's address (make it before any stream
 * capture).  Returned errors never carry a message; a CUDA failure inside the
 * transform is also recorded, with its text, for zk_last_error(). */
ZK_EXTERN RustError zk_lde_noalloc(void *d_output, const void *d_input, uint32_t lg_n, uint32_t rate_bits,
                                   uint32_t batches, uint32_t inv, uint32_t with_coset, void *stream);

/* ---- batched and served commits (no counterpart in zeknox) ---- */

/* One commit job on device buffers: coefficients batches x 2^lg_n; outputs
 * leaves 2^(lg_n+rate_bits) x batches (leaf layout), digests
 * 2*(N - 2^cap_height) x 4, cap 2^cap_height x 4. */
typedef struct {
    const void *d_coeffs;
    uint32_t lg_n, rate_bits, batches, cap_height, hash_type;
    void *d_leaves, *d_digests, *d_cap;
} ZkCommitJob;

/* All jobs, stream-ordered on `stream`: forked onto n_streams internal streams
 * (0 = 4), largest jobs first onto the least-loaded stream, joined back.  Each
 * job's outputs equal zk_commit_async's. */
ZK_EXTERN RustError zk_commit_batch(const ZkCommitJob *jobs, uint32_t n_jobs, uint32_t n_streams, void *stream);

/* Autotuner of a commit shape (commits, batches, the server): for one shape
 * (2^lg_n coefficients, rate_bits, batches polynomials) it times, on scratch
 * data, every legal pass count (2 or 3) and polynomials-per-block of the
 * LDE -> leaves pass, and for Poseidon trees of up to 2^16 leaves the six-,
 * two- and one-thread-per-hash leaf kernels; it keeps the fastest of each for
 * that shape class, and later commits of the class use them.  Outputs do not
 * depend on the choices.  Synchronous: call outside stream capture.  *timed
 * receives the number of candidates timed (0: already tuned, or nothing to
 * tune).  zk_autotune_reset forgets every choice. */
ZK_EXTERN RustError zk_autotune_commit(uint32_t lg_n, uint32_t rate_bits, uint32_t batches, int32_t *timed);
ZK_EXTERN RustError zk_autotune_reset(void);

/* Commit server: jobs are submitted with host coefficients (kept valid by the
 * caller until the job completes), admitted onto n_slots concurrent streams
 * while leaves + digests + cap of resident trees plus coefficients + scratch of
 * running jobs fit hbm_budget_bytes, and keep their tree on the device until
 * released.  Admission is first in, first out, except that a later, shorter
 * job may start ahead of or beside earlier ones when its estimated GPU time
 * fits in each of their delay budgets (a twentieth of each one's own
 * estimated GPU time, from job sizes; ZK_SERVER_BUDGET_FRAC overrides the
 * fraction), which it then uses up.
 * zk_server_wait blocks until the cap is on the host.
 * zk_server_wait_any returns, in completion order, each job that has finished
 * (or failed) since the last call, once; *ticket = 0 when nothing is pending or
 * when timeout_ms passes first (UINT32_MAX waits without limit).  The server
 * keeps its own memory pool and reserves hbm_budget_bytes (plus an eighth for
 * fragmentation) in it when it is created; each slot's worker thread
 * allocates and launches the jobs admitted to it. */
typedef struct ZkServer ZkServer;
typedef struct {
    uint64_t completed, queued, max_queue;
    double p50_s, p99_s, max_s; /* submit -> cap on the host */
    double elems, elems_per_s;  /* committed LDE evaluations; first submit -> last completion */
    uint64_t hbm_in_use, hbm_peak;
    uint64_t ahead; /* jobs started ahead of an older queued job or beside a running one */
    double alloc_max_s; /* longest host time one job's device allocations took */
    uint64_t pool_reserved_start; /* bytes the server's memory pool mapped at creation */
    uint64_t pool_reserved_high;  /* most bytes it has mapped since (above the first: it grew) */
} ZkServerStats;
ZK_EXTERN RustError zk_server_create(int32_t device, uint64_t hbm_budget_bytes, uint32_t n_slots, ZkServer **out);
ZK_EXTERN RustError zk_server_submit(ZkServer *srv, const void *host_coeffs, uint32_t lg_n, uint32_t rate_bits,
                                     uint32_t batches, uint32_t cap_height, uint32_t hash_type, uint64_t *ticket);
/* A job whose coefficients (batches x 2^lg_n) are the field-element stream
 * zk_fill_field_async(seed) writes, generated on the device when the job is
 * admitted instead of copied from the host: a load source for measuring the
 * server with device-resident inputs. */
ZK_EXTERN RustError zk_server_submit_seeded(ZkServer *srv, uint64_t seed, uint32_t lg_n, uint32_t rate_bits,
                                            uint32_t batches, uint32_t cap_height, uint32_t hash_type,
                                            uint64_t *ticket);
ZK_EXTERN RustError zk_server_wait(ZkServer *srv, uint64_t ticket, uint64_t *host_cap, double *latency_s);
ZK_EXTERN RustError zk_server_wait_any(ZkServer *srv, uint32_t timeout_ms, uint64_t *ticket);
ZK_EXTERN RustError zk_server_result(ZkServer *srv, uint64_t ticket, void **d_leaves, void **d_digests,
                                     void **d_cap);
ZK_EXTERN RustError zk_server_release(ZkServer *srv, uint64_t ticket);
ZK_EXTERN RustError zk_server_stats(ZkServer *srv, ZkServerStats *out);
/* Where a completed job's latency went (before zk_server_release): submit ->
 * start (queued_s) and start -> cap on the host (run_s). */
ZK_EXTERN RustError zk_server_job_times(ZkServer *srv, uint64_t ticket, double *queued_s, double *run_s);
/* Host-side fault injection for tests: the next n_jobs admitted jobs fail at
 * their at_allocation-th device allocation (1 = coefficients, 2 = leaves,
 * 3 = digests, ...) as if the pool were exhausted.  A failed job reports its
 * error through zk_server_wait; its partial allocations are freed and the
 * server keeps serving. */
ZK_EXTERN RustError zk_server_inject_failure(ZkServer *srv, uint32_t n_jobs, uint32_t at_allocation);
ZK_EXTERN RustError zk_server_destroy(ZkServer *srv);

#endif /* ZEKNOX_B200_H */
