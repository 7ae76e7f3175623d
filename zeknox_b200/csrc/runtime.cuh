// Host runtime of the library: error type, per-device context (stream,
// twiddle / coset tables), and a few launch helpers.
//
// Replaces zeknox's sppark-derived gpu_t / stream_t / dev_ptr_t
// (native/utils/gpu_t.cuh:82-486) and CUDA_OK / cuda_error
// (native/utils/exception.cuh:13-23) for the one-GPU path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace zk {

// A failure carried to the C ABI boundary: `code` becomes RustError.code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char *what, const char *file, int line);

#define ZK_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t zk_e_ = (call);                                            \
        if (zk_e_ != cudaSuccess) ::zk::throw_cuda(zk_e_, #call, __FILE__, __LINE__); \
    } while (0)

// Every kernel launch of the library goes through ZK_CHECK_LAUNCH, which also
// counts it (zk_kernel_launches() in the C ABI).
void note_launch();
#define ZK_CHECK_LAUNCH()                \
    do {                                 \
        ZK_CUDA(cudaGetLastError());     \
        ::zk::note_launch();             \
    } while (0)

uint64_t launch_count();

// Records a failure on this thread for zk_last_error() (capi.cu).
void record_last_error(int code, const char *msg);

inline void require(bool ok, const std::string &msg) {
    if (!ok) throw Error((int)cudaErrorInvalidValue, msg);
}

// ---- field helpers on the host (table construction) ----
constexpr uint64_t P_HOST = 0xffffffff00000001ull;
inline uint64_t h_mul(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) % P_HOST); }
inline uint64_t h_pow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    a %= P_HOST;
    while (e) {
        if (e & 1) r = h_mul(r, a);
        a = h_mul(a, a);
        e >>= 1;
    }
    return r;
}
inline uint64_t h_inv(uint64_t a) { return h_pow(a, P_HOST - 2); }
// Primitive 2^lg-th root of unity: 7^((p-1)/2^lg) (zeknox native/ff/gl64_params.hpp:15).
inline uint64_t h_omega(unsigned lg) { return h_pow(7, (P_HOST - 1) >> lg); }
constexpr uint64_t GROUP_GENERATOR = 7;  // native/ff/gl64_params.hpp:12

// Two-level power table of a base b:  b^e = lo[e & (2^h - 1)] * hi[e >> h]
// for e < 2^bits.  Both halves live in one device allocation.
struct PowTable {
    uint64_t *dev = nullptr;  // [lo (2^h) | hi (2^(bits-h))]
    uint64_t *full = nullptr; // b^e for every e < 2^bits when bits <= kFullTableMaxLg, else null
    unsigned bits = 0, h = 0;
    uint64_t base = 0;
    const uint64_t *lo() const { return dev; }
    const uint64_t *hi() const { return dev + (1ull << h); }
};

constexpr int kMaxLg = 32;
constexpr unsigned kFullTableMaxLg = 20;  // one-load power tables up to 2^20 entries (8 MB)
constexpr int kLineLgMax = 12;  // longest in-shared-memory line: 4096 elements

// Per-device state.  Tables are built lazily, under `mu`.
struct DeviceCtx {
    int dev = -1;
    cudaStream_t stream = nullptr;       // blocking stream (orders after the legacy stream)
    cudaStream_t copy_stream = nullptr;  // host<->device copies overlapped with `stream`
    cudaStream_t lane_stream = nullptr;  // second compute lane of the host-buffer LDE
    uint64_t *line_roots[2] = {nullptr, nullptr};  // [dir] omega_4096^j, j < 4096
    PowTable roots[2][kMaxLg + 1];       // [dir][lg]: omega_{2^lg} powers
    PowTable coset;                      // coset_gen powers
    std::map<std::pair<uint64_t, unsigned>, PowTable> shifts;  // other bases (base, bits), kept until exit
    std::mutex mu;
};

DeviceCtx &device_ctx(int dev);
int current_device();
int device_count();

// Tables (created on first use; the returned references stay valid).
const uint64_t *line_roots(DeviceCtx &c, bool inverse);
const PowTable &root_table(DeviceCtx &c, unsigned lg, bool inverse);
// Coset powers for at least 2^lg points.  A request with a different
// generator replaces the table (init_coset semantics); a larger lg extends it.
const PowTable &coset_table(DeviceCtx &c, unsigned lg, uint64_t gen, bool replace);
// Powers of an arbitrary base for 2^bits exponents, built once per (base, bits)
// and never replaced (the shifted cosets of FRI rounds use these).
const PowTable &shift_table(DeviceCtx &c, unsigned bits, uint64_t base);
// The coset generator the coset LDEs of device `dev` use: the one init_coset
// installed last, GROUP_GENERATOR before that.  A plain read of a per-device
// word (no context or table is created), for the allocation-free LDE.
uint64_t installed_coset_generator(int dev);

// Stream-ordered scratch from the device's default memory pool.
struct Scratch {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    Scratch() = default;
    Scratch(size_t bytes, cudaStream_t st) { alloc(bytes, st); }
    void alloc(size_t bytes, cudaStream_t st) {
        s = st;
        if (bytes && !p) ZK_CUDA(cudaMallocAsync(&p, bytes, st));
    }
    ~Scratch() {
        if (p) cudaFreeAsync(p, s);
    }
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
    template <class T>
    T *as() const { return (T *)p; }
};

}  // namespace zk
