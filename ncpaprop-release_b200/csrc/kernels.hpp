// Launchers of the sm_100a kernels of the ESS normal-mode path.  Host code in
// ncpa_api.cu calls these; each returns the number of kernels it launched.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ncpa {

// error flags written by kernels into the context's device status word
enum : unsigned {
    kErrTimeout = 1u,  // a bounded mbarrier wait gave up
    kErrBracket = 2u,  // bisection bracket inconsistent with the Sturm counts
    kErrWkb = 4u,      // WKB search needed more trial wavenumbers than threads
    kErrTooMany = 8u,  // a problem has more modes than allowed (device-built work items)
};

// Per (frequency, azimuth) problem, device resident.  Every problem carries
// its own solver grid (size, spacing, source/receiver rows and the offsets of
// its rows in the batch arrays), so one batch may mix grid sizes.
struct ProblemInfo {
    double freq, omega, az;
    double k_min, k_max;   // wavenumber window [1/m]
    double lo, hi;         // window in units of the scaled matrix S = h^2 A
    double ceff_grnd, ceff_top;
    double dz;             // grid spacing [m]
    unsigned long long ceffmin_bits, ceffmax_bits;  // positive doubles as ordered bits
    long long s_off;       // offset (doubles) of the problem's row in s, g and kz2 (rows padded to kChunk)
    long long w_off;       // offset (doubles) of its attenuation-weight row in w
    int nz;                // grid points
    int isrc, ircv;        // source / receiver grid rows
    int c_lo, c_hi;        // Sturm counts at lo, hi
    int M, off;            // number of modes and offset into the mode arrays
    int used_wkb;
    int n_scan;            // shifts of the isolation scan (<= kScanMax)
    int n_scan_raw;        // the size estimated from the problem alone (before the batch-wide trim)
    float m_est;           // estimated mode count in [lo, hi] (-1: not estimated)
    double g0;             // wide-angle rows: ground term of row 0, 1 / (dz admittance + 1)
};

struct WorkItem {
    int problem;  // problem index
    int j0;       // first eigen-index inside the problem (0 = lowest k)
    int m;        // eigenvalues in this item (<= kWItem for bisection)
    int pad;
};

constexpr int kScanMax = 512;      // count slots per problem of the isolation scan
constexpr int kScanDefault = 256;  // shifts per problem unless the scan sizes them (wide-angle rows)
constexpr int kChunk = 1024;      // doubles per TMA chunk of the diagonal
constexpr int kBlk = 16;          // eigenvector checkpoint interval
constexpr int kCkRows = 128;      // twist candidates of the reduction-only eigenvector items
// elements of each eigenvector checkpoint array per warp slot for grids of up
// to nz points: q every kBlk rows (items that write full vectors) or three
// sums every kCkRows rows (items that only reduce)
inline long long ck_slot_elems(long long nz) {
    const long long a = (nz + kBlk - 1) / kBlk, b = 3 * ((nz + kCkRows - 1) / kCkRows);
    return (a > b ? a : b) * 32;
}
constexpr int kThreads = 256;     // threads of the scan CTAs
constexpr int kWItem = 32;        // eigenvalues per warp work item of the bisection
constexpr int kEvItem = 32;       // eigenvalues per warp work item of the eigenvector kernel
constexpr int kEvWarpsPerCta = 4; // warps per eigenvector CTA
// bisection item scheduler state (ints): ticket, heavy-end and light-end
// counters, then one arrival counter per (SM < kSchedSms, sub-partition)
constexpr int kSchedSms = 256;
constexpr int kSchedInts = 3 + 4 * kSchedSms;
constexpr int kSchedWorkers = 2;  // default bisection warps per warp scheduler

// knot-level derived quantities
int launch_steffen(cudaStream_t st, int n, const double* x, const double* y, int batch, int ystride,
                   double* coef, int cstride);
int launch_profile_derived(cudaStream_t st, int n, const double* z, const double* u, const double* v,
                           const double* p, const double* rho, const double* pcoef, const double* rcoef,
                           int have_c0, double* c0, double* ws, double* wd);
int launch_ceff_knots(cudaStream_t st, int n, int n_az, const double* az, const double* c0, const double* ws,
                      const double* wd, double* ceff);
int launch_alpha_knots(cudaStream_t st, int n, int n_f, const double* freqs, const double* z, const double* t,
                       const double* p, const double* rho, double* alpha);
// grid sampling of the frequency-independent fields: rho, P on the grid and
// c_T = sqrt(1.4 P / rho)
int launch_grid_common(cudaStream_t st, int nk, const double* zk, const double* rho, const double* rcoef,
                       const double* p, const double* pcoef, int nz, double z_min, double dz_grid,
                       double* rho_g, double* ct_g);
// attenuation weight w = 2 alpha omega / c_T for every frequency [n_f x nz]
int launch_attn_weight(cudaStream_t st, int nk, const double* zk, const double* alpha, const double* acoef,
                       int n_f, const double* freqs, int nz, double z_min, double dz_grid, const double* ct_g,
                       double* w, int wstride);
// matrix build (K1): s, optional kz2 = (omega/c)^2 and g = 1/c^2, each
// [P x nz_pad]; fills ceff extrema / ground / top in ProblemInfo (the P
// problems of one launch share one grid; their rows are nz_pad apart)
int launch_build_matrix(cudaStream_t st, int nk, const double* zk, const double* ceffk, const double* ceffcoef,
                        int n_az, int P, ProblemInfo* pinfo, int nz, int nz_pad, double z_min, double dz_grid,
                        double dz, double admittance, double* s, double* kz2, double* g);
// WKB window and scaled bounds (K2)
int launch_window(cudaStream_t st, int P, ProblemInfo* pinfo, const double* kz2, int wkb, int wvnum,
                  double c_min, double c_max, unsigned* err);
// isolation scan (K3a): sizes each problem's scan (ProblemInfo::n_scan) from
// an estimate of its mode count, then pinfo[p].n_scan Sturm counts per
// problem at counts[p * kScanMax + t]
// slots > 0 (warp schedulers of the device: 4 x SMs) trims the batch's scan
// to a whole number of units per scheduler; sched (kSchedInts ints, zeroed)
// then has the units claimed per scheduler (see k_scan)
int launch_scan(cudaStream_t st, int P, ProblemInfo* pinfo, const double* s, int* counts, unsigned* err,
                int slots = 0, int* sched = nullptr);
// multisection/bisection over work items (K3); step_counter (optional)
// accumulates the Sturm recurrence steps swept; sched (kSchedInts ints,
// zeroed) runs a cost-ordered item list (order = 1 in launch_make_items) with
// `workers` warps per warp scheduler (the first from the heavy end of the
// list, the others from the light end); null maps items round-robin
int launch_bisect(cudaStream_t st, int grid, const ProblemInfo* pinfo, const double* s, const int* counts,
                  const WorkItem* items, int n_items, int* counter, double tol, double* mu, unsigned* err,
                  unsigned long long* step_counter, const int* n_items_dev = nullptr, int* sched = nullptr,
                  int workers = kSchedWorkers);
int bisect_ctas_per_sm();
// FP64 throughput probe: each thread runs n_iter iterations of 8 independent
// FMA chains; out receives a value that keeps the chains live
int launch_fp64_probe(cudaStream_t st, int grid, int block, int n_iter, double* out);
// twisted-factorisation eigenvectors + fused reductions (K4)
struct EigvecArgs {
    const ProblemInfo* pinfo;
    const double* s;   // rows at pinfo[p].s_off
    const double* w;   // rows at pinfo[p].w_off
    const double* g;   // rows at pinfo[p].s_off, or null
    const WorkItem* items;
    int n_items;
    const int* n_items_dev;  // when set, the item count is read here (built on the device)
    const int* ev_done;      // when set, items with ev_done[it] != 0 are skipped (done in the fused launch)
    int* counter;
    const double* mu;
    double* kr;
    double* ki;
    double* vs;
    double* vr;
    double* vg;
    double* vfull;            // optional: per problem [nz x M] at vfull_off[p]
    const long long* vfull_off;
    double* ck_q1;            // checkpoint scratch, one slot per warp of the grid
    double* ck_q2;
    int* ck_e;
    long long ck_slot_stride; // elements per warp slot (blocks of the largest grid x 32)
    unsigned* err;
};
int launch_eigvec(cudaStream_t st, int grid, const EigvecArgs& a);
// Bisection and eigenvectors in one launch (ESS rows, no group speeds, no
// full vectors): bisection items as launch_bisect, then eigenvector items of
// finished problems from a ready queue.  pstat[3 P] from k_make_items;
// queue[ev_cap], q_head, q_tail and ev_done[ev_cap] zeroed before the launch.
// A k_eigvec launch with ea.ev_done = ev_done must follow: it runs the items
// this launch did not finish.
struct FusedArgs {
    int P;
    const ProblemInfo* pinfo;
    const double* s;
    const int* counts;
    const WorkItem* bis;
    const int* n_bis_dev;
    double tol;
    double* mu;
    unsigned* err;
    int* pstat;
    int* queue;
    int* q_head;
    int* q_tail;
    int* ev_done;
    unsigned long long wait_ns;  // a consumer gives up on an empty slot after this long
    int* sched;                  // bisection item scheduler (kSchedInts, zeroed) or null (round-robin)
    int workers;                 // bisection warps per warp scheduler with sched
    int ev_workers_only;         // only warps that ran bisection take eigenvector items
    EigvecArgs ea;
};
int launch_bisect_eigvec(cudaStream_t st, int grid, const FusedArgs& a);
int fused_ctas_per_sm();
// the same on the wide-angle rows (mu = kappa; follow with launch_eigvec_wmod)
int launch_bisect_eigvec_wmod(cudaStream_t st, int grid, const FusedArgs& a);
int fused_wmod_ctas_per_sm();
// Work items built on the device from the Sturm scan: per problem c_lo, c_hi,
// M and CSR offset in pinfo; bisection items (<= bis_item eigenvalues, sizes
// balanced inside a problem) and eigenvector items (kEvItem) appended;
// tot = {n_bisect_items, n_eigvec_items, total modes}.  Sets kErrTooMany if a
// problem exceeds max_modes (its M is then clamped) or a capacity is exceeded.
// pstat (optional, 3 P ints): per problem the number of bisection items, the
// first eigenvector item and the number of eigenvector items.  order = 1
// lists the bisection items by estimated cost, heaviest problems first (for
// P <= 4096; problem order otherwise)
int launch_make_items(cudaStream_t st, int P, ProblemInfo* pinfo, const int* counts, int max_modes, int bis_item,
                      WorkItem* bis_items, int bis_cap, WorkItem* ev_items, int ev_cap, int* tot, unsigned* err,
                      int* pstat = nullptr, int order = 0);
// resident eigenvector CTAs per SM for the variant selected by a
int eigvec_ctas_per_sm(const EigvecArgs& a);
// modal sums
int launch_tl1d(cudaStream_t st, int P, const ProblemInfo* pinfo, const double* kr, const double* ki,
                const double* vs, const double* vr, int nr, double dr, int lossless, double* re, double* im,
                double* incoh);
int launch_tl2d(cudaStream_t st, int M, const double* kr, const double* ki, const double* vs_src,
                const double* vz, int nzo, int nr, double dr, int lossless, double* re, double* im);
// same sum with [n_rcv x nr] output (receiver-major)
int launch_tl2d_rcv_major(cudaStream_t st, int M, const double* kr, const double* ki, const double* vs_src,
                          const double* vz, int n_rcv, int nr, double dr, int lossless, double* re, double* im);
// out[c][r] = in[r][c] (rows x cols doubles)
int launch_transpose(cudaStream_t st, int rows, int cols, const double* in, double* out);
// broadband synthesis
int launch_twiddle(cudaStream_t st, int nfft, double* tw);
// fac: scratch of 4 doubles per mode
int launch_bb_transfer(cudaStream_t st, int nfreq, const int* off, const double* re_k, const double* im_k,
                       const double* vs, const double* vr, double rho_ratio, int nr, const double* ranges,
                       int zero_attn, int n_modes, double* fac, double* h);
int launch_src_builtin(cudaStream_t st, int kind, int nfreq, const double* f, double scale, double* out);
int launch_spline_eval(cudaStream_t st, int n, const double* x, const double* y, const double* coef, int m,
                       const double* xq, double* out);
int launch_starter(cudaStream_t st, int M, int nz, int step, int isrc, const double* v, const double* kr,
                   double k0, double* out);
int launch_fill_unit(cudaStream_t st, int n, double* h);
int launch_src_pulse2(cudaStream_t st, int n, double dt, double scale, double* x);
int launch_bb_pulse(cudaStream_t st, int nfreq, const double* f, const double* s_src, const double* h, int nr,
                    const double* t0, int nfft, const double* tw, double* out);
int launch_src_dft(cudaStream_t st, int n, const double* x, double dt, int nfft, int nfreq, const double* tw,
                   double* s);

// Wide-angle (WMod) modes (wmod.cu).  Rows of T(k) h^2 in the WmodRows
// format (device_common.cuh): two doubles per row, (B_i, U_i) interleaved, at
// 2 * pinfo[p].s_off (the s layout, rows padded to kChunk); row 0's ground
// term goes to pinfo[p].g0.  The eigen-solve runs in kappa = h k: pinfo
// k_min / k_max bound the window in k, kappa_min = k_min dz.
int launch_wc_knots(cudaStream_t st, int n, int n_az, const double* az, const double* ws, const double* wd,
                    double* wc);
int launch_wmod_build(cudaStream_t st, int nk, const double* zk, const double* c0k, const double* c0c,
                      const double* wck, const double* wcc, const double* ceffk, const double* ceffc, int n_az,
                      int P, ProblemInfo* pinfo, int nz, int nz_pad, double z_min, double dz_grid, double dz,
                      double admittance, double* rows, double* kz2);
int launch_wscan(cudaStream_t st, int P, const ProblemInfo* pinfo, const double* rows, int* counts, unsigned* err);
// k_bisect on the wide-angle rows: mu receives kappa = h k; tol is relative
// to kappa_max; step_counter (optional) counts chain steps (3 FMA each) as
// launch_bisect does
int launch_bisect_wmod(cudaStream_t st, int grid, const ProblemInfo* pinfo, const double* rows, const int* counts,
                       const WorkItem* items, double tol, double* mu, unsigned* err,
                       unsigned long long* step_counter, const int* n_items_dev, int* sched = nullptr,
                       int workers = kSchedWorkers);
int bisect_wmod_ctas_per_sm();
// eigenvectors of the wide-angle rows: EigvecArgs with s = rows, mu = kappa,
// g = null; vectors normalised to sum v^2 dz = 1 / (1 + k^2)
int launch_eigvec_wmod(cudaStream_t st, int grid, const EigvecArgs& a);
int eigvec_wmod_ctas_per_sm(const EigvecArgs& a);

// K5 modal sum on the tensor cores (modal_sum.cu)
struct MsPlan {
    int groups, n_chunks, M_pad, n_tiles, n_ctas, n_parts;
    long long n_units;  // (receiver group, range tile, mode chunk) units
    size_t a_img_bytes, q_bytes, tab_bytes, raw_bytes;
    // guarded sum (fmt 2): partial sums of |A'|, FP64 tables, flagged points
    size_t s_part_bytes, b64_bytes, tp64_bytes, a64_bytes, fix_list_bytes;
};
MsPlan ms_plan(int n_rcv, int M, int n_ranges, int num_sms);
// flag threshold of the guarded sum: a point with |P| < tau S is recomputed
double ms_guard_tau(const MsPlan& p);
// the error bound eps behind it: |P_tc - P| <= eps S
double ms_guard_eps(const MsPlan& p);
int launch_ms_gather(cudaStream_t st, int n_rcv, int M, const int* idx, const double* vfull, double* vz);
// fmt: 0 = 3-term split-BF16 (kind::f16), 1 = TF32 (kind::tf32), 2 = guarded
// 6-term split-BF16.  Buffers: a_img = A as complex FP32 per (receiver group,
// mode chunk), q = tile phases, tab = the B' image of each mode chunk
// (tile-independent); b64, tp64, a64 (fmt 2 only, else NULL) = the FP64
// offset phases, tile phases and A the fix-up reads
int launch_ms_prepare(cudaStream_t st, const MsPlan& p, int fmt, int n_rcv, int M, const double* kr,
                      const double* ki, const double* vs, const int* idx, const double* vfull, double dr, int lossless,
                      void* a_img, void* q, void* tab, void* b64, void* tp64, void* a64);
// variant: the schedule (ring depths) of the tensor-core kernel, 0 ..
// ms_tc_variants() - 1 (0: the deepest rings); results do not depend on it
int launch_ms_tc(cudaStream_t st, const MsPlan& p, int fmt, int n_ranges, const void* a_img, const void* q,
                 const void* tab, float* raw, float* s_part, unsigned* err, int variant);
int ms_tc_variants();
// ranges per tile of the tensor-core sums (the UMMA N)
int ms_tile_ranges();
void ms_tc_variant_shape(int fmt, int variant, int* t_stages, int* g_stages);
// s_part non-NULL: flag the points the guarded sum must recompute into
// fix_list / fix_count (zeroed by the caller)
int launch_ms_finish(cudaStream_t st, const MsPlan& p, int n_rcv, int n_ranges, double dr, const float* raw,
                     double* re, double* im, const float* s_part, int* fix_count, void* fix_list);
int launch_ms_fix(cudaStream_t st, int num_sms, int M, int M_pad, int n_ranges, double dr, const int* fix_count,
                  const void* fix_list, const void* a64, const void* tp64, const void* b64, double* re, double* im);

}  // namespace ncpa
