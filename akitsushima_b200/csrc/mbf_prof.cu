// Launch profiler and device peak probes.
#include <mutex>
#include <string>
#include <vector>

#include "mbf_util.cuh"

namespace mbf {

bool g_prof_on = false;

struct ProfRec {
    std::string name;
    cudaEvent_t a, b;
};

static std::mutex g_prof_mu;
static std::vector<ProfRec> g_prof;
static std::vector<cudaEvent_t> g_pool;

static cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void prof_mark(const char *name, cudaStream_t st, bool start) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (start) {
        ProfRec r;
        r.name = name;
        r.a = take_event();
        r.b = nullptr;
        cudaEventRecord(r.a, st);
        g_prof.push_back(r);
    } else {
        for (auto it = g_prof.rbegin(); it != g_prof.rend(); ++it) {
            if (it->b == nullptr && it->name == name) {
                it->b = take_event();
                cudaEventRecord(it->b, st);
                break;
            }
        }
    }
}

// FMA-chain probe: each thread runs independent chains of a*x+b; the
// result is written so the compiler keeps the work.
template <typename T>
__global__ void fma_probe(T *out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x * T(1e-3), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

}  // namespace mbf

using namespace mbf;

extern "C" {

void mbf_profile_begin(void) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto &r : g_prof) {
        g_pool.push_back(r.a);
        if (r.b) g_pool.push_back(r.b);
    }
    g_prof.clear();
    g_prof_on = true;
}

// Writes "name count total_ms\n" lines into buf (NUL-terminated); returns the
// number of kernels listed, or a negative code.
int mbf_profile_end(char *buf, size_t cap) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_on = false;
    if (cudaDeviceSynchronize() != cudaSuccess) return MBF_ERR_CUDA;
    std::vector<std::string> names;
    std::vector<double> tot;
    std::vector<int> cnt;
    for (auto &r : g_prof) {
        if (!r.b) continue;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        size_t k = 0;
        for (; k < names.size(); ++k)
            if (names[k] == r.name) break;
        if (k == names.size()) {
            names.push_back(r.name);
            tot.push_back(0.0);
            cnt.push_back(0);
        }
        tot[k] += ms;
        cnt[k] += 1;
    }
    std::string out;
    for (size_t k = 0; k < names.size(); ++k) {
        char line[256];
        snprintf(line, sizeof line, "%s %d %.9f\n", names[k].c_str(), cnt[k], tot[k]);
        out += line;
    }
    if (buf && cap > 0) {
        size_t n = out.size() < cap - 1 ? out.size() : cap - 1;
        memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return (int)names.size();
}

// Sustained FMA throughput of this GPU in FLOP/s (2 per FMA) for float64
// (precision 0) or float32 (1), timed with events over `reps` launches.
int mbf_peak_probe(int precision, void *scratch, size_t scratch_bytes, double *flops, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0, n_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    int block = 256, grid = n_sm * 8, iters = 4096;
    size_t need = (size_t)grid * block * sizeof(double);
    if (!scratch || scratch_bytes < need || !flops) return MBF_ERR_ARGUMENT;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    auto launch = [&]() {
        if (precision == MBF_FP64)
            fma_probe<double><<<grid, block, 0, st>>>((double *)scratch, iters, 0.999999, 1e-7);
        else
            fma_probe<float><<<grid, block, 0, st>>>((float *)scratch, iters, 0.999999f, 1e-7f);
    };
    launch();
    cudaEventRecord(a, st);
    const int reps = 5;
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(b, st);
    if (cudaEventSynchronize(b) != cudaSuccess) return MBF_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    double fl = 2.0 * 8 * 16 * (double)iters * grid * block * reps;
    *flops = fl / (ms * 1e-3);
    return MBF_OK;
}

}  // extern "C"
