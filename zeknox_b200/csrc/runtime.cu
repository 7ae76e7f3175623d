// Per-device context and table construction (host side).
#include <stdio.h>

#include <atomic>
#include <memory>

#include "runtime.cuh"

namespace zk {

void throw_cuda(cudaError_t e, const char *what, const char *file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
    // zeknox reports CUDA failures as -cudaError (native/utils/exception.cuh:22).
    throw Error(-(int)e, buf);
}

namespace {
std::atomic<uint64_t> g_launches{0};
}
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

int current_device() {
    int d = 0;
    ZK_CUDA(cudaGetDevice(&d));
    return d;
}

int device_count() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

namespace {
std::mutex g_ctx_mu;
std::vector<std::unique_ptr<DeviceCtx>> g_ctx;

// Upload a host vector to a fresh device allocation (synchronous; tables are small).
uint64_t *upload(const std::vector<uint64_t> &v) {
    uint64_t *d = nullptr;
    ZK_CUDA(cudaMalloc(&d, v.size() * sizeof(uint64_t)));
    ZK_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
    return d;
}

PowTable make_pow_table(uint64_t base, unsigned bits) {
    PowTable t;
    t.base = base;
    t.bits = bits;
    t.h = (bits + 1) / 2;
    const uint64_t nlo = 1ull << t.h, nhi = 1ull << (bits - t.h);
    std::vector<uint64_t> v(nlo + nhi);
    uint64_t x = 1;
    for (uint64_t i = 0; i < nlo; i++, x = h_mul(x, base)) v[i] = x;  // x = base^nlo at exit
    const uint64_t step = x;
    uint64_t y = 1;
    for (uint64_t i = 0; i < nhi; i++, y = h_mul(y, step)) v[nlo + i] = y;
    t.dev = upload(v);
    if (bits <= kFullTableMaxLg) {
        std::vector<uint64_t> f(1ull << bits);
        uint64_t z = 1;
        for (auto &e : f) {
            e = z;
            z = h_mul(z, base);
        }
        t.full = upload(f);
    }
    return t;
}
}  // namespace

DeviceCtx &device_ctx(int dev) {
    std::lock_guard<std::mutex> g(g_ctx_mu);
    if (g_ctx.empty()) {
        int n = device_count();
        if (n <= 0) throw Error((int)cudaErrorNoDevice, "no CUDA device available");
        g_ctx.resize(n);
    }
    if (dev < 0 || dev >= (int)g_ctx.size())
        throw Error((int)cudaErrorInvalidDevice, "invalid device id " + std::to_string(dev));
    if (!g_ctx[dev]) {
        auto c = std::make_unique<DeviceCtx>();
        c->dev = dev;
        ZK_CUDA(cudaSetDevice(dev));
        // Blocking stream: work on it is ordered after the legacy default stream,
        // like zeknox's per-GPU "zero" stream (native/utils/gpu_t.cuh:246-252).
        ZK_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault));
        ZK_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        ZK_CUDA(cudaStreamCreateWithFlags(&c->lane_stream, cudaStreamNonBlocking));
        // Keep freed pool memory cached between calls.
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        g_ctx[dev] = std::move(c);
    }
    return *g_ctx[dev];
}

const uint64_t *line_roots(DeviceCtx &c, bool inv) {
    std::lock_guard<std::mutex> g(c.mu);
    if (!c.line_roots[inv]) {
        uint64_t w = h_omega(kLineLgMax);
        if (inv) w = h_inv(w);
        std::vector<uint64_t> v(1u << kLineLgMax);
        uint64_t x = 1;
        for (auto &e : v) {
            e = x;
            x = h_mul(x, w);
        }
        c.line_roots[inv] = upload(v);
    }
    return c.line_roots[inv];
}

const PowTable &root_table(DeviceCtx &c, unsigned lg, bool inv) {
    require(lg >= 1 && lg <= (unsigned)kMaxLg, "transform size 2^" + std::to_string(lg) + " out of range");
    std::lock_guard<std::mutex> g(c.mu);
    PowTable &t = c.roots[inv][lg];
    if (!t.dev) {
        uint64_t w = h_omega(lg);
        t = make_pow_table(inv ? h_inv(w) : w, lg);
    }
    return t;
}

namespace {
constexpr int kGenDevices = 64;
std::atomic<uint64_t> g_coset_gen[kGenDevices];  // 0: none installed yet
}  // namespace

uint64_t installed_coset_generator(int dev) {
    const uint64_t g = (dev >= 0 && dev < kGenDevices) ? g_coset_gen[dev].load(std::memory_order_acquire) : 0;
    return g ? g : GROUP_GENERATOR;
}

const PowTable &coset_table(DeviceCtx &c, unsigned lg, uint64_t gen, bool replace) {
    std::lock_guard<std::mutex> g(c.mu);
    PowTable &t = c.coset;
    // Without `replace` an existing generator is kept (the LDE uses whatever
    // init_coset installed, as zeknox does); a larger size extends the table.
    const uint64_t want_gen = (t.dev && !replace) ? t.base : gen;
    unsigned want_bits = lg < 2 ? 2 : lg;
    if (t.dev && t.base == want_gen && t.bits > want_bits) want_bits = t.bits;
    if (!t.dev || t.base != want_gen || t.bits < want_bits) {
        if (t.dev) {
            ZK_CUDA(cudaDeviceSynchronize());  // no kernel may still read the old table
            cudaFree(t.dev);
            if (t.full) cudaFree(t.full);
            t.dev = t.full = nullptr;
        }
        t = make_pow_table(want_gen, want_bits);
    }
    if (c.dev >= 0 && c.dev < kGenDevices) g_coset_gen[c.dev].store(t.base, std::memory_order_release);
    return t;
}

const PowTable &shift_table(DeviceCtx &c, unsigned bits, uint64_t base) {
    require(bits <= (unsigned)kMaxLg, "shift table of 2^" + std::to_string(bits) + " powers out of range");
    if (bits < 2) bits = 2;
    base %= P_HOST;
    std::lock_guard<std::mutex> g(c.mu);
    PowTable &t = c.shifts[{base, bits}];  // std::map: references stay valid as it grows
    if (!t.dev) t = make_pow_table(base, bits);
    return t;
}

}  // namespace zk
