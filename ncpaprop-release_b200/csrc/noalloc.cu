// Allocation-free eigenvector entry point (ncpa_eigvec_static in
// include/ncpa_gpu.h).
//
// Who needs it: callers that must not allocate device memory once they run --
// for instance a host application that sizes and reserves all GPU memory at
// start-up, a code path that runs inside a stream-ordered memory budget it
// does not own, or an embedding runtime whose allocator cannot be re-entered
// from the thread that calls us.  ncpa_ess_solve allocates its temporaries;
// this entry point computes the eigenvectors, the perturbative attenuation
// and the source / receiver mode values of one problem for eigenvalues the
// caller already has, using only the caller's buffers and one fixed scratch
// array that lives in the library image.
//
// The scratch is the file-scope array g_eigvec_scratch below
// (kStaticScratchBytes, about 21 MiB).  Every GPU that loads the library holds
// it until the process exits.  All calls share it: a call overwrites what the
// previous call left there, and calls whose work overlaps on the GPU (two
// streams, two host threads) race on it.  The first call on a device looks up
// the array's device address with cudaGetSymbolAddress (once per device, with
// that device current); make that first call before any stream capture.
// The address is kept for the life of the process: after cudaDeviceReset on a
// device the library image is loaded anew there, so a process that resets a
// device must not call this entry point on it again.  Every call waits for its
// own work to finish before it returns (it reads the device error word back
// and synchronises the stream).
#include <cstdint>
#include <mutex>

#include "kernels.hpp"
#include "ncpa_gpu.h"

namespace {

using ncpa::ProblemInfo;
using ncpa::WorkItem;

constexpr int kStaticMaxNz = 32768;        // grid points
constexpr int kStaticMaxModes = 4000;      // eigenvalues per call
constexpr int kStaticWarps = 16;           // eigenvector warps (4 CTAs)
constexpr int kStaticChunk = 256;          // padding of the diagonal copies
constexpr int kStaticBlocks = kStaticMaxNz / ncpa::kBlk;
static_assert((long long)kStaticBlocks * 32 >= 3LL * ((kStaticMaxNz + ncpa::kCkRows - 1) / ncpa::kCkRows) * 32,
              "checkpoint slots cover the coarse sums of the largest grid");
constexpr int kStaticItems = (kStaticMaxModes + ncpa::kEvItem - 1) / ncpa::kEvItem;

// byte layout of the scratch array
constexpr size_t kOffS = 0;                                                  // s copy [kStaticMaxNz]
constexpr size_t kOffW = kOffS + (size_t)kStaticMaxNz * 8;                    // w copy [kStaticMaxNz]
constexpr size_t kCkElems = (size_t)kStaticWarps * kStaticBlocks * 32;        // checkpoint elements
constexpr size_t kOffQ1 = kOffW + (size_t)kStaticMaxNz * 8;
constexpr size_t kOffQ2 = kOffQ1 + kCkElems * 8;
constexpr size_t kOffE = kOffQ2 + kCkElems * 8;
constexpr size_t kOffItems = (kOffE + kCkElems * 4 + 255) / 256 * 256;
constexpr size_t kOffInfo = (kOffItems + (size_t)kStaticItems * sizeof(WorkItem) + 255) / 256 * 256;
constexpr size_t kOffCounter = (kOffInfo + sizeof(ProblemInfo) + 255) / 256 * 256;  // int counter, unsigned err
constexpr size_t kStaticScratchBytes = kOffCounter + 256;

static_assert(kStaticMaxNz % kStaticChunk == 0, "padding");

}  // namespace

// The scratch array.  Host code must not use its name as a device address;
// the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_eigvec_scratch[kStaticScratchBytes];

namespace {

// copies the caller's diagonal and weights into the padded scratch copies and
// writes the work list, the problem record and zeroed counters
__global__ void k_static_setup(unsigned char* base, const double* __restrict__ s, const double* __restrict__ w,
                               int nz, int n, double omega, double lo, double dz, int isrc, int ircv) {
    double* sc = reinterpret_cast<double*>(base + kOffS);
    double* wc = reinterpret_cast<double*>(base + kOffW);
    const int nz_pad = (nz + kStaticChunk - 1) / kStaticChunk * kStaticChunk;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nz_pad; i += gridDim.x * blockDim.x) {
        sc[i] = i < nz ? s[i] : 0.0;
        wc[i] = i < nz ? w[i] : 0.0;
    }
    if (blockIdx.x == 0) {
        WorkItem* items = reinterpret_cast<WorkItem*>(base + kOffItems);
        const int n_items = (n + ncpa::kEvItem - 1) / ncpa::kEvItem;
        for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
            const int j0 = it * ncpa::kEvItem;
            items[it] = WorkItem{0, j0, min(ncpa::kEvItem, n - j0), 0};
        }
        if (threadIdx.x == 0) {
            ProblemInfo* pi = reinterpret_cast<ProblemInfo*>(base + kOffInfo);
            *pi = ProblemInfo{};
            pi->omega = omega;
            pi->lo = lo;
            pi->dz = dz;
            pi->nz = nz;
            pi->isrc = isrc;
            pi->ircv = ircv;
            pi->s_off = 0;
            pi->w_off = 0;
            pi->M = n;
            pi->off = 0;
            int* counter = reinterpret_cast<int*>(base + kOffCounter);
            counter[0] = 0;
            reinterpret_cast<unsigned*>(counter)[1] = 0u;
        }
    }
}

std::mutex g_setup_mutex;
void* g_scratch_ptr[256];  // device address of g_eigvec_scratch, per device ordinal

}  // namespace

extern "C" ncpa_status ncpa_eigvec_static(const double* s, const double* w, int nz, double dz, const double* mu,
                                          int n_modes, int isrc, int ircv, double omega, double* re_k,
                                          double* im_k, double* v_src, double* v_rcv, void* stream) {
    if (!s || !w || !mu || !re_k || !im_k || !v_src || !v_rcv) return NCPA_EINVAL;
    if (nz < 3 || nz > kStaticMaxNz) return NCPA_EINVAL;          // grid beyond the scratch
    if (n_modes < 1 || n_modes > kStaticMaxModes) return NCPA_ETOOMANY;
    if (isrc < 0 || isrc >= nz || ircv < 0 || ircv >= nz || !(dz > 0.0)) return NCPA_EINVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return NCPA_ENODEV;
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_eigvec_scratch) != cudaSuccess || !p) return NCPA_ECUDA;
            g_scratch_ptr[dev] = p;
        }
        base = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nz_pad = (nz + kStaticChunk - 1) / kStaticChunk * kStaticChunk;
    k_static_setup<<<(nz_pad + 255) / 256, 256, 0, st>>>(base, s, w, nz, n_modes, omega, 0.0, dz, isrc,
                                                             ircv);
    if (cudaGetLastError() != cudaSuccess) return NCPA_ECUDA;
    ncpa::EigvecArgs a{};
    a.pinfo = reinterpret_cast<const ProblemInfo*>(base + kOffInfo);
    a.s = reinterpret_cast<const double*>(base + kOffS);
    a.w = reinterpret_cast<const double*>(base + kOffW);
    a.g = nullptr;
    a.items = reinterpret_cast<const WorkItem*>(base + kOffItems);
    a.n_items = (n_modes + ncpa::kEvItem - 1) / ncpa::kEvItem;
    a.counter = reinterpret_cast<int*>(base + kOffCounter);
    a.mu = mu;
    a.kr = re_k;
    a.ki = im_k;
    a.vs = v_src;
    a.vr = v_rcv;
    a.vg = nullptr;
    a.vfull = nullptr;
    a.vfull_off = nullptr;
    a.ck_q1 = reinterpret_cast<double*>(base + kOffQ1);
    a.ck_q2 = reinterpret_cast<double*>(base + kOffQ2);
    a.ck_e = reinterpret_cast<int*>(base + kOffE);
    a.ck_slot_stride = ncpa::ck_slot_elems(nz);
    a.err = reinterpret_cast<unsigned*>(base + kOffCounter) + 1;
    ncpa::launch_eigvec(st, kStaticWarps / ncpa::kEvWarpsPerCta, a);
    if (cudaGetLastError() != cudaSuccess) return NCPA_ECUDA;
    unsigned herr = 0;
    if (cudaMemcpyAsync(&herr, a.err, sizeof herr, cudaMemcpyDeviceToHost, st) != cudaSuccess) return NCPA_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return NCPA_ECUDA;
    if (herr == 0u) return NCPA_OK;
    // a ring wait that gave up is a timeout; any other device error bit is not
    return (herr & ~ncpa::kErrTimeout) ? NCPA_ECUDA : NCPA_ETIMEDOUT;
}
