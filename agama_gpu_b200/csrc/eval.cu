// eval.cu -- the fused per-point kernel and the C ABI (include/agb.h).
//
// One thread per point (grid-stride).  Each thread reads its position once,
// walks the leaves (component + Shifted/Scaled/Evolving transform) in order,
// evaluates each component in its own frame and accumulates
//   Phi += A Phi_c,  grad += A sigma grad_c,  H/rho += A sigma^2 (H_c/rho_c)
// in FP64, then writes the outputs once.  This replaces the reference's chain
// of one launch per component plus CuPy elementwise passes for shifts, scales,
// negation, lerps and sums (gpu_potential.py:1439-1918).
#include <cuda.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <stdio.h>
#include <string.h>
#include <stdarg.h>
#include <stdlib.h>
#include "agb_dev.cuh"
#include "multipole.cuh"
#include "cylspline.cuh"
#include "analytic.cuh"
#include "bin.cuh"
#include "mp_grad.cuh"
#include "cs_grad.cuh"
#include "adjoint_steps.cuh"
#include "time_plan.cuh"

// ---------------------------------------------------------------------------
// errors and launch accounting
// ---------------------------------------------------------------------------
static thread_local char g_err[512] = "";
static thread_local long long g_launches = 0;

static int set_err(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

extern "C" const char* agb_last_error(void) { return g_err; }
extern "C" const char* agb_version(void) { return "agama_gpu_b200 0.1 (sm_100a)"; }
extern "C" int64_t agb_launch_count(void) { return g_launches; }
extern "C" void agb_launch_count_reset(void) { g_launches = 0; }

static int check_launch(const char* what)
{
    ++g_launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_err(AGB_ERR_DEVICE, "%s: launch failed: %s", what, cudaGetErrorString(e));
    return AGB_OK;
}

// ---------------------------------------------------------------------------
// the fused kernel
// ---------------------------------------------------------------------------
// AN: the tree holds analytic leaves only (no expansion code compiled in: a
// small register footprint and more resident blocks for the Hessian modes)
template <int MODE, typename R, bool EXACT, bool AN = false>
__device__ __forceinline__ void eval_component(const DevComp& c, double x, double y, double z,
                                               PointOut& o)
{
    switch (c.kind) {
    case AGB_KIND_MULTIPOLE:     if (!AN) multipole_point<MODE, R>(c, x, y, z, o); break;
    case AGB_KIND_CYLSPLINE:     if (!AN) cylspline_point<MODE, EXACT, R>(c, x, y, z, o); break;
    case AGB_KIND_NFW:           nfw_point<MODE>(c.p, x, y, z, o); break;
    case AGB_KIND_PLUMMER:       plummer_point<MODE>(c.p, x, y, z, o); break;
    case AGB_KIND_HERNQUIST:     hernquist_point<MODE>(c.p, x, y, z, o); break;
    case AGB_KIND_DEHNEN:        dehnen_point<MODE>(c.p, x, y, z, o); break;
    case AGB_KIND_ISOCHRONE:     isochrone_point<MODE>(c.p, x, y, z, o); break;
    case AGB_KIND_MIYAMOTONAGAI: mn_point<MODE>(c.p, x, y, z, o); break;
    case AGB_KIND_LOGHALO:       loghalo_point<MODE>(c.p, x, y, z, o); break;
    case AGB_KIND_DISKANSATZ:    diskansatz_point<MODE>(c.p, x, y, z, o); break;
    case AGB_KIND_UNIFORMACC:    uniform_point<MODE>(c.p, x, y, z, o); break;
    default: break;
    }
}

// Binned calls evaluate the points in interval order.  Writing each point's
// outputs straight to its input position scatters 8-byte stores over the whole
// output (uncoalesced: one sector per lane per store); with room in the
// workspace the kernel instead writes records in sorted order ("stage") and
// unpermute_kernel gathers them back, reading one record per point and writing
// every output array contiguously.
// internal mode of agb_eval_vjp_force: the VJP plus the force of the same leaves
// (written to the `hess` pointer as [N,3]) from the same per-point sums
#define AGB_MODE_VJPF 5

__host__ __device__ constexpr int stage_rec(int mode)
{
    return mode == AGB_MODE_HESS ? 10 : mode == AGB_MODE_GRAD ? 4 : mode == AGB_MODE_VJP ? 3
         : mode == AGB_MODE_VJPF ? 6 : 1;
}
#define AGB_STAGE_MAX_REC 10

template <int MODE>
__global__ void __launch_bounds__(256)
unpermute_kernel(const int* __restrict__ dest, const double* __restrict__ stage, long long n,
                 double* phi, double* grad, double* hess, double* rho)
{
    constexpr int REC = stage_rec(MODE);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double* t = stage + (long long)REC * __ldg(dest + i);
        if (MODE == AGB_MODE_DENS) { rho[i] = t[0]; continue; }
        if (MODE == AGB_MODE_VJP || MODE == AGB_MODE_VJPF) {
            grad[3 * i] = t[0]; grad[3 * i + 1] = t[1]; grad[3 * i + 2] = t[2];
            if (MODE == AGB_MODE_VJPF) {
                hess[3 * i] = t[3]; hess[3 * i + 1] = t[4]; hess[3 * i + 2] = t[5];
            }
            continue;
        }
        if (phi) phi[i] = t[0];
        if (MODE != AGB_MODE_POT && grad) {
            grad[3 * i] = t[1]; grad[3 * i + 1] = t[2]; grad[3 * i + 2] = t[3];
        }
        if (MODE == AGB_MODE_HESS) {
            #pragma unroll
            for (int q = 0; q < 6; ++q) hess[6 * i + q] = t[4 + q];
        }
    }
}

// Hessian-carrying modes hold about twice the live state: one block per SM
// with up to 255 registers beats two blocks with heavy spilling.
// analytic-only Hessian modes: 3 blocks per SM (80 registers) measured 1.2 % faster per
// backward leapfrog step than 2 (and than 4, which spills more)
// DYN: the leaves come from device memory (agb_eval_timed: computed by
// time_leaves_kernel from a device-resident time), copied to shared memory once
// per block; otherwise they are kernel parameters.
// BS: threads per block (AGB_OUT_BLOCK); the resident-block bound scales with it so
// that every block size keeps the register budget of the 256-thread shape.
__host__ __device__ constexpr int eval_min_blocks(int mode, bool an, int bs)
{
    return (((mode == AGB_MODE_HESS || mode == AGB_MODE_VJP || mode == AGB_MODE_VJPF) && !an)
            ? 1 : (an ? 3 : 2)) * 256 / bs;
}

template <int MODE, typename R, bool AN = false, bool DYN = false, int BS = 256>
__global__ void __launch_bounds__(BS, eval_min_blocks(MODE, AN, BS))
agb_eval_kernel(const __grid_constant__ EvalArgs a)
{
    // the VJP modes evaluate every component with its Hessian and contract at the end
    constexpr bool VJP = MODE == AGB_MODE_VJP || MODE == AGB_MODE_VJPF;
    constexpr int CM = VJP ? AGB_MODE_HESS : MODE;
    __shared__ DevLeaf dyn_leaves[DYN ? AGB_MAX_LEAVES : 1];
    if (DYN) {
        for (int q = threadIdx.x; q < a.n_leaves; q += blockDim.x) dyn_leaves[q] = a.dleaves[q];
        __syncthreads();
    }
    // a contiguous range of (interval-sorted) points per block: consecutive
    // iterations of a block reuse the same interval's table records from L1
    const long long lo = (long long)blockIdx.x * a.chunk;
    const long long hi = lo + a.chunk < a.n ? lo + a.chunk : a.n;
    for (long long pos = lo + threadIdx.x; pos < hi; pos += blockDim.x) {
        double x, y, z;
        if (a.soa) {
            x = a.x[pos]; y = a.y[pos]; z = a.z[pos];
        } else {
            x = a.xyz[3 * pos]; y = a.xyz[3 * pos + 1]; z = a.xyz[3 * pos + 2];
        }
        const long long i = a.perm ? (long long)a.perm[pos] : pos;
        double phi = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, rho = 0.0;
        double h[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int L = 0; L < a.n_leaves; ++L) {
            const DevLeaf& lf = DYN ? dyn_leaves[L] : a.leaves[L];
            // a zero-weight leaf (the unused snapshot of an Evolving bracket at a snapshot
            // time) contributes nothing: skipped, so its partner is walked alone, as the
            // host flattening evaluates it
            if (lf.ampl == 0.0) continue;
            const DevComp& c = a.comps[lf.comp];
            const double lx = lf.sigma * x - lf.g0;
            const double ly = lf.sigma * y - lf.g1;
            const double lz = lf.sigma * z - lf.g2;
            if ((MODE == AGB_MODE_POT || MODE == AGB_MODE_GRAD) && !AN &&
                std::is_same<R, float>::value && lf.pad == 1 &&
                (DYN ? dyn_leaves[L + 1] : a.leaves[L + 1]).ampl != 0.0) {
                // this leaf and the next share grid, columns and transform (pack_args);
                // FP32 walks only (the FP64 walk holds twice the state and would spill)
                const DevLeaf& lf2 = DYN ? dyn_leaves[L + 1] : a.leaves[L + 1];
                PointOut o1, o2;
                o1.phi = o2.phi = 0.0;
                o1.g[0] = o1.g[1] = o1.g[2] = 0.0;
                o2.g[0] = o2.g[1] = o2.g[2] = 0.0;
                multipole_pair_point<CM, R>(c, a.comps[lf2.comp], lx, ly, lz, o1, o2);
                phi += lf.ampl * o1.phi;
                phi += lf2.ampl * o2.phi;
                if (CM != AGB_MODE_POT) {
                    const double As1 = lf.ampl * lf.sigma, As2 = lf2.ampl * lf2.sigma;
                    g0 += As1 * o1.g[0]; g1 += As1 * o1.g[1]; g2 += As1 * o1.g[2];
                    g0 += As2 * o2.g[0]; g1 += As2 * o2.g[1]; g2 += As2 * o2.g[2];
                }
                ++L;
                continue;
            }
            PointOut o;
            o.phi = 0.0; o.rho = 0.0;
            o.g[0] = o.g[1] = o.g[2] = 0.0;
            #pragma unroll
            for (int q = 0; q < 6; ++q) o.h[q] = 0.0;
            eval_component<CM, R, VJP, AN>(c, lx, ly, lz, o);
            const double A = lf.ampl;
            if (CM == AGB_MODE_DENS) {
                rho += (A * lf.sigma * lf.sigma) * o.rho;
                continue;
            }
            phi += A * o.phi;
            if (CM != AGB_MODE_POT) {
                const double As = A * lf.sigma;
                g0 += As * o.g[0]; g1 += As * o.g[1]; g2 += As * o.g[2];
                if (CM == AGB_MODE_HESS) {
                    const double As2 = As * lf.sigma;
                    #pragma unroll
                    for (int q = 0; q < 6; ++q) h[q] += As2 * o.h[q];
                }
            }
        }
        if (VJP) {
            // L(Phi, F): dL/dx = gPhi grad(Phi) + (dF/dx)^T gF = gPhi grad(Phi) - H gF
            const double gp = a.gphi ? a.gphi[i] : 0.0;
            double f0 = 0.0, f1 = 0.0, f2 = 0.0;
            if (a.gforce) { f0 = a.gforce[3 * i]; f1 = a.gforce[3 * i + 1]; f2 = a.gforce[3 * i + 2]; }
            const double v0 = gp * g0 - (h[0] * f0 + h[3] * f1 + h[5] * f2);
            const double v1 = gp * g1 - (h[3] * f0 + h[1] * f1 + h[4] * f2);
            const double v2 = gp * g2 - (h[5] * f0 + h[4] * f1 + h[2] * f2);
            if (MODE == AGB_MODE_VJPF) {
                if (a.stage) {
                    double* o = a.stage + 6 * pos;
                    o[0] = v0; o[1] = v1; o[2] = v2; o[3] = -g0; o[4] = -g1; o[5] = -g2;
                } else {
                    a.grad[3 * i] = v0; a.grad[3 * i + 1] = v1; a.grad[3 * i + 2] = v2;
                    a.hess[3 * i] = -g0; a.hess[3 * i + 1] = -g1; a.hess[3 * i + 2] = -g2;
                }
                continue;
            }
            double* o = a.stage ? a.stage + 3 * pos : a.grad + 3 * i;
            o[0] = v0; o[1] = v1; o[2] = v2;
            continue;
        }
        const double sg = (a.out_flags & AGB_OUT_NEGATE) ? -1.0 : 1.0;
        if (MODE == AGB_MODE_DENS) {
            if (a.stage) a.stage[pos] = rho;
            else a.rho[i] = rho;
            continue;
        }
        if (a.stage) {
            // sorted order: consecutive threads write consecutive records
            constexpr int REC = stage_rec(MODE);
            double* o = a.stage + REC * pos;
            o[0] = phi;
            if (MODE != AGB_MODE_POT) { o[1] = sg * g0; o[2] = sg * g1; o[3] = sg * g2; }
            if (MODE == AGB_MODE_HESS) {
                #pragma unroll
                for (int q = 0; q < 6; ++q) o[4 + q] = sg * h[q];
            }
            continue;
        }
        if (a.phi) a.phi[i] = phi;
        if (MODE != AGB_MODE_POT && a.grad) {
            a.grad[3 * i] = sg * g0; a.grad[3 * i + 1] = sg * g1; a.grad[3 * i + 2] = sg * g2;
        }
        if (MODE == AGB_MODE_HESS) {
            #pragma unroll
            for (int q = 0; q < 6; ++q) a.hess[6 * i + q] = sg * h[q];
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Values fixed for the life of a device (its SM count, the resident blocks of one
// kernel) are read on the device current at the call and cached per device index.
// Host threads making their first call at the same time store the same value, so
// relaxed atomics are enough.
#define AGB_MAX_DEVICES 64

static int current_device()
{
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= AGB_MAX_DEVICES) d = 0;
    return d;
}

static std::atomic<int> g_num_sms[AGB_MAX_DEVICES];

static int num_sms()
{
    const int dev = current_device();
    int v = g_num_sms[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        g_num_sms[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// resident blocks per SM of `kernel` at `threads` threads, cached per device in `cache`
template <typename K>
static int blocks_per_sm(std::atomic<int>* cache, K kernel, int threads)
{
    const int dev = current_device();
    int b = cache[dev].load(std::memory_order_relaxed);
    if (b == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, 0) != cudaSuccess || b < 1)
            b = 1;
        cache[dev].store(b, std::memory_order_relaxed);
    }
    return b;
}

static int grid_for(long long n)
{
    const long long blocks = (n + 255) / 256;
    const long long cap = (long long)num_sms() * 64;
    return (int)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

// blocks per resident slot.  Measured on the 4M-point composite (mixed): 1 wave (the
// largest contiguous chunk per block, most L1 reuse of an interval's records) is best
// for one large launch, 4.86 ms against 4.99 ms with 4; for the 0.25-1M-point launches
// of the host pipeline 2 waves give the shortest end-to-end step (6.44 against 6.72 ms).
static int default_waves(long long n) { return n > (1LL << 21) ? 1 : 2; }

// resident blocks per SM of one instantiation
template <int MODE, typename R, bool AN, bool DYN = false, int BS = 256>
static int eval_blocks_per_sm()
{
    static std::atomic<int> per_sm[AGB_MAX_DEVICES];
    return blocks_per_sm(per_sm, agb_eval_kernel<MODE, R, AN, DYN, BS>, BS);
}

// points that one wave of resident threads holds (one point per thread)
template <int MODE, typename R, bool AN = false>
static long long eval_wave_points()
{
    return (long long)num_sms() * eval_blocks_per_sm<MODE, R, AN>() * 256;
}

// The launch shape.  Each block takes one contiguous range of a.chunk points:
// AGB_OUT_PPT(p) fixes the range at BS x 2^(p-1) points (points per thread) and
// the grid grows with n; otherwise the grid is AGB_OUT_GRID's blocks per resident
// slot (default_waves when unset) and the range is what the points need.
template <int MODE, typename R, bool AN, bool DYN, int BS>
static void launch_eval_bs(EvalArgs& a, cudaStream_t st)
{
    const int p = (a.out_flags >> AGB_OUT_PPT_SHIFT) & 15;
    long long grid;
    if (p) {
        long long chunk = (long long)BS << (p - 1);
        if ((a.n + chunk - 1) / chunk > 0x7fffffffLL)      // the grid's x limit
            chunk = ((a.n + 0x7ffffffeLL) / 0x7fffffffLL + 31) / 32 * 32;
        a.chunk = chunk;
        grid = (a.n + chunk - 1) / chunk;
        if (grid < 1) grid = 1;
    } else {
        const int per_sm = eval_blocks_per_sm<MODE, R, AN, DYN, BS>();
        const long long want = (a.n + BS - 1) / BS;
        const int w = (a.out_flags >> AGB_OUT_GRID_SHIFT) & 15;
        const long long slots = (long long)num_sms() * per_sm * (w ? w : default_waves(a.n));
        grid = want < slots ? (want > 0 ? want : 1) : slots;
        a.chunk = ((a.n + grid - 1) / grid + 31) / 32 * 32;
    }
    agb_eval_kernel<MODE, R, AN, DYN, BS><<<(int)grid, BS, 0, st>>>(a);
}

// AGB_OUT_BLOCK picks 128 or 512 threads per block for the host-leaf kernels of
// the four evaluation modes; 512 only where the 256-thread shape holds two blocks
// per SM (the Hessian kernel's 255 registers a thread leave room for 256 threads).
// Device-time leaves, the analytic-only and the VJP kernels run 256 threads.
template <int MODE, typename R, bool AN = false, bool DYN = false>
static void launch_eval(EvalArgs& a, cudaStream_t st)
{
    constexpr bool SHAPES = !AN && !DYN && MODE != AGB_MODE_VJP && MODE != AGB_MODE_VJPF;
    int b = (a.out_flags >> AGB_OUT_BLOCK_SHIFT) & 3;
    // the default shape of large force calls of trees with a Multipole: 512 threads per
    // block, one block per SM.  Measured on the 4M-point composite, binned step: mixed
    // 4.18 -> 4.06 ms, FP64 7.02 -> 6.77 ms against 256 threads x 2 blocks per SM
    const int shape_bits = (15 << AGB_OUT_GRID_SHIFT) | (15 << AGB_OUT_PPT_SHIFT);
    // and of large Hessian calls: 128 threads per block, FP32 walk one block per slot
    // (8.50 -> 8.22 ms), FP64 16 points per thread (11.34 -> 11.06 ms)
    // and of large density calls: 512 threads (mixed 4.80 -> 4.64 ms, FP64 7.78 -> 7.37 ms)
    if ((MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS) && b == 0 &&
        !(a.out_flags & shape_bits) && a.n > (1LL << 21)) {
        bool mp = false;
        for (int L = 0; L < a.n_leaves && !mp; ++L)
            mp = a.comps[a.leaves[L].comp].kind == AGB_KIND_MULTIPOLE;
        if (mp && (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_DENS)) b = 2;
        if (mp && MODE == AGB_MODE_HESS) {
            b = 1;
            if (std::is_same<R, double>::value) a.out_flags |= 5 << AGB_OUT_PPT_SHIFT;
        }
    }
    if constexpr (SHAPES) {
        if (b == 1) return launch_eval_bs<MODE, R, AN, DYN, 128>(a, st);
        if constexpr (eval_min_blocks(MODE, AN, 256) >= 2)
            if (b == 2) return launch_eval_bs<MODE, R, AN, DYN, 512>(a, st);
    }
    launch_eval_bs<MODE, R, AN, DYN, 256>(a, st);
}

static bool analytic_only(const EvalArgs& a)
{
    for (int L = 0; L < a.n_leaves; ++L) {
        const int k = a.comps[a.leaves[L].comp].kind;
        if (k == AGB_KIND_MULTIPOLE || k == AGB_KIND_CYLSPLINE) return false;
    }
    return true;
}

static int launch_eval_mode(int mode, int precision, EvalArgs& a, cudaStream_t st);

template <int MODE>
static void launch_unpermute(const EvalArgs& a, cudaStream_t st)
{
    unpermute_kernel<MODE><<<grid_for(a.n), 256, 0, st>>>(a.dest, a.stage, a.n, a.phi, a.grad,
                                                          a.hess, a.rho);
}

static int launch_mode(int mode, int precision, EvalArgs& a, cudaStream_t st)
{
    int rc = launch_eval_mode(mode, precision, a, st);
    if (rc || !a.stage) return rc;
    switch (mode) {
    case AGB_MODE_POT:  launch_unpermute<AGB_MODE_POT>(a, st); break;
    case AGB_MODE_GRAD: launch_unpermute<AGB_MODE_GRAD>(a, st); break;
    case AGB_MODE_HESS: launch_unpermute<AGB_MODE_HESS>(a, st); break;
    case AGB_MODE_DENS: launch_unpermute<AGB_MODE_DENS>(a, st); break;
    case AGB_MODE_VJPF: launch_unpermute<AGB_MODE_VJPF>(a, st); break;
    default:            launch_unpermute<AGB_MODE_VJP>(a, st); break;
    }
    return check_launch("unpermute_kernel");
}

static int launch_eval_mode(int mode, int precision, EvalArgs& a, cudaStream_t st)
{
    const bool mixed = precision == AGB_PREC_MIXED;
    if (a.dleaves) {        // leaves computed on the device (agb_eval_timed)
        switch (mode) {
        case AGB_MODE_POT:  mixed ? launch_eval<AGB_MODE_POT, float, false, true>(a, st)  : launch_eval<AGB_MODE_POT, double, false, true>(a, st); break;
        case AGB_MODE_GRAD: mixed ? launch_eval<AGB_MODE_GRAD, float, false, true>(a, st) : launch_eval<AGB_MODE_GRAD, double, false, true>(a, st); break;
        case AGB_MODE_HESS: mixed ? launch_eval<AGB_MODE_HESS, float, false, true>(a, st) : launch_eval<AGB_MODE_HESS, double, false, true>(a, st); break;
        case AGB_MODE_DENS: mixed ? launch_eval<AGB_MODE_DENS, float, false, true>(a, st) : launch_eval<AGB_MODE_DENS, double, false, true>(a, st); break;
        default: return set_err(AGB_ERR_ARG, "agb_eval_timed: mode %d is not supported", mode);
        }
        return check_launch("agb_eval_kernel");
    }
    switch (mode) {
    case AGB_MODE_POT:  mixed ? launch_eval<AGB_MODE_POT, float>(a, st)  : launch_eval<AGB_MODE_POT, double>(a, st); break;
    case AGB_MODE_GRAD: mixed ? launch_eval<AGB_MODE_GRAD, float>(a, st) : launch_eval<AGB_MODE_GRAD, double>(a, st); break;
    case AGB_MODE_HESS: mixed ? launch_eval<AGB_MODE_HESS, float>(a, st) : launch_eval<AGB_MODE_HESS, double>(a, st); break;
    case AGB_MODE_DENS: mixed ? launch_eval<AGB_MODE_DENS, float>(a, st) : launch_eval<AGB_MODE_DENS, double>(a, st); break;
    // analytic leaves compute in FP64 in both precisions: one lean instantiation
    case AGB_MODE_VJP:
        if (analytic_only(a)) launch_eval<AGB_MODE_VJP, double, true>(a, st);
        else mixed ? launch_eval<AGB_MODE_VJP, float>(a, st) : launch_eval<AGB_MODE_VJP, double>(a, st);
        break;
    case AGB_MODE_VJPF:
        if (analytic_only(a)) launch_eval<AGB_MODE_VJPF, double, true>(a, st);
        else mixed ? launch_eval<AGB_MODE_VJPF, float>(a, st) : launch_eval<AGB_MODE_VJPF, double>(a, st);
        break;
    default: return set_err(AGB_ERR_ARG, "agb_eval: unknown mode %d", mode);
    }
    return check_launch("agb_eval_kernel");
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

static int comp_to_dev(const agb_component& s, DevComp& d, int precision)
{
    memset(&d, 0, sizeof(d));
    d.kind = s.kind;
    d.n_lm = s.n_lm; d.n_int = s.n_int; d.nz = s.nz; d.lmax = s.lmax;
    d.log_scaling = s.log_scaling; d.layout = s.layout; d.lm_split = 0;
    d.structure = s.structure;
    d.table = s.table; d.table32 = s.table32; d.lm = s.lm; d.lm_m = nullptr;
    d.grid_a = s.grid_a; d.grid_b = s.grid_b; d.extra = s.extra;
    memcpy(d.p, s.p, sizeof(d.p));
    if (s.kind == AGB_KIND_MULTIPOLE) {
        if (!s.table || !s.lm || s.n_lm < 1 || s.n_int < 1)
            return set_err(AGB_ERR_ARG, "multipole component: missing table/lm or empty sizes");
        if (s.lmax > AGB_MAX_LMAX)
            return set_err(AGB_ERR_UNSUPPORTED, "multipole lmax=%d exceeds %d", s.lmax, AGB_MAX_LMAX);
        if (!aligned16(s.table))
            return set_err(AGB_ERR_ARG, "multipole table must be 16-byte aligned");
        if (s.structure < AGB_STRUCT_LIST || s.structure > AGB_STRUCT_EVEN)
            return set_err(AGB_ERR_ARG, "multipole structure %d unknown", s.structure);
        if (s.structure != AGB_STRUCT_LIST) {
            if (s.layout != AGB_LAYOUT_INTERVAL_MAJOR)
                return set_err(AGB_ERR_ARG, "regular multipole tables must be interval-major");
            int cols = 0;
            for (int m = 0; m <= s.lmax; ++m)
                for (int l = m; l <= s.lmax; ++l)
                    if (s.structure == AGB_STRUCT_ALL || (l % 2) == 0) cols += (m == 0) ? 1 : 2;
            if (cols != s.n_lm)
                return set_err(AGB_ERR_ARG, "regular multipole table: n_lm=%d, structure needs %d columns",
                               s.n_lm, cols);
        }
        if (precision == AGB_PREC_MIXED) {
            if (!s.table32 || !aligned16(s.table32))
                return set_err(AGB_ERR_ARG, "mixed precision needs a 16-byte aligned FP32 table");
        }
    } else if (s.kind == AGB_KIND_CYLSPLINE) {
        if (!s.table || !s.lm || !s.grid_a || !s.grid_b || !s.extra || s.n_int < 2 || s.nz < 2)
            return set_err(AGB_ERR_ARG, "cylspline component: missing tables or grid < 2 nodes");
        if (!aligned16(s.table))
            return set_err(AGB_ERR_ARG, "cylspline table must be 16-byte aligned");
        if (s.lmax > AGB_MAX_LMAX || (int)s.p[2] > s.lmax)
            return set_err(AGB_ERR_ARG, "cylspline outer multipole orders out of range");
        if (precision == AGB_PREC_MIXED && s.table32 && !aligned16(s.table32))
            return set_err(AGB_ERR_ARG, "cylspline FP32 table must be 16-byte aligned");
    } else if (s.kind < AGB_KIND_NFW || s.kind > AGB_KIND_UNIFORMACC) {
        return set_err(AGB_ERR_ARG, "unknown component kind %d", s.kind);
    }
    return AGB_OK;
}

// Binning plan: the Multipole leaf with the most harmonics keys the sort.
struct BinPlan {
    bool on;
    BinKey key;
    int n_bins;
    int leaf;          // the keyed leaf
};

static BinPlan plan_binning(const agb_component* comps, const agb_leaf* leaves, int n_leaves,
                            int64_t n, int out_flags)
{
    BinPlan b;
    memset(&b, 0, sizeof(b));
    if ((out_flags & AGB_OUT_NO_BINNING) || n > 0x7fffffffLL) return b;
    if (n < AGB_BIN_MIN_POINTS && !(out_flags & AGB_OUT_BIN_ALWAYS)) return b;
    int best = -1, best_lm = 0;
    for (int L = 0; L < n_leaves; ++L) {
        const agb_component& c = comps[leaves[L].comp];
        if (c.kind == AGB_KIND_MULTIPOLE && c.n_lm > best_lm && c.n_int + 2 <= AGB_MAX_BINS) {
            best = L;
            best_lm = c.n_lm;
        }
    }
    if (best < 0 || best_lm < 2) return b;
    const agb_component& c = comps[leaves[best].comp];
    b.on = true;
    b.leaf = best;
    b.key.sigma = leaves[best].sigma;
    b.key.g0 = leaves[best].gamma[0]; b.key.g1 = leaves[best].gamma[1]; b.key.g2 = leaves[best].gamma[2];
    b.key.logr_min = c.p[0];
    b.key.inv_dlogr = c.p[2];
    b.key.n_int = c.n_int;
    // output blocks of 2^19 points (40 MB of Hessian output at most), more
    // points per block when the block count would exceed the bin limit
    const int nb = c.n_int + 2;
    int lb = 19;
    while ((long long)((n + (1LL << lb) - 1) >> lb) * nb > AGB_MAX_BINS) ++lb;
    b.key.log_block = lb;
    b.n_bins = (int)((n + (1LL << lb) - 1) >> lb) * nb;
    return b;
}

static constexpr size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t ws_bytes(const BinPlan& b, int64_t n)
{
    if (!b.on) return 0;
    return al256(4 * (size_t)n) * 2 + al256(24 * (size_t)n) + al256(4 * (size_t)b.n_bins) * 2;
}

// with room for the sorted-order output records (stage_rec doubles per point)
static size_t ws_bytes_staged(const BinPlan& b, int64_t n)
{
    if (!b.on) return 0;
    return ws_bytes(b, n) + al256(8 * (size_t)AGB_STAGE_MAX_REC * (size_t)n);
}

static int validate(const agb_component* comps, int n_comps, const agb_leaf* leaves, int n_leaves,
                    const double* xyz, int64_t n, int mode, int precision, double* phi,
                    double* grad, double* hess, double* rho)
{
    if (n < 0) return set_err(AGB_ERR_ARG, "agb_eval: negative point count");
    if (n > 0 && !xyz) return set_err(AGB_ERR_ARG, "agb_eval: xyz is null");
    if (!comps || n_comps < 1 || !leaves || n_leaves < 1)
        return set_err(AGB_ERR_ARG, "agb_eval: empty component or leaf list");
    if (n_leaves > AGB_MAX_LEAVES)
        return set_err(AGB_ERR_UNSUPPORTED, "agb_eval: %d leaves exceed %d", n_leaves, AGB_MAX_LEAVES);
    for (int L = 0; L < n_leaves; ++L)
        if (leaves[L].comp < 0 || leaves[L].comp >= n_comps || leaves[L].comp >= 256)
            return set_err(AGB_ERR_ARG, "agb_eval: leaf %d refers to component %d of %d", L,
                           leaves[L].comp, n_comps);
    if (precision != AGB_PREC_FP64 && precision != AGB_PREC_MIXED)
        return set_err(AGB_ERR_ARG, "agb_eval: unknown precision %d", precision);
    switch (mode) {
    case AGB_MODE_POT:  if (!phi) return set_err(AGB_ERR_ARG, "agb_eval: phi is null"); break;
    case AGB_MODE_GRAD: if (!grad) return set_err(AGB_ERR_ARG, "agb_eval: grad is null"); break;
    case AGB_MODE_HESS: if (!hess) return set_err(AGB_ERR_ARG, "agb_eval: hess is null"); break;
    case AGB_MODE_DENS: if (!rho) return set_err(AGB_ERR_ARG, "agb_eval: rho is null"); break;
    case AGB_MODE_VJP:  if (!grad) return set_err(AGB_ERR_ARG, "agb_eval_vjp: g_xyz is null"); break;
    case AGB_MODE_VJPF:
        if (!grad || !hess) return set_err(AGB_ERR_ARG, "agb_eval_vjp_force: g_xyz or force is null");
        break;
    default: return set_err(AGB_ERR_ARG, "agb_eval: unknown mode %d", mode);
    }
    return AGB_OK;
}

static int pack_args(EvalArgs& a, const agb_component* comps, int n_comps, const agb_leaf* leaves,
                     int n_leaves, int precision)
{
    int remap[256];
    for (int i = 0; i < 256; ++i) remap[i] = -1;
    int nc = 0;
    for (int L = 0; L < n_leaves; ++L) {
        const int ci = leaves[L].comp;
        if (remap[ci] < 0) {
            if (nc >= AGB_MAX_COMPONENTS)
                return set_err(AGB_ERR_UNSUPPORTED, "agb_eval: more than %d distinct components", AGB_MAX_COMPONENTS);
            const int rc = comp_to_dev(comps[ci], a.comps[nc], precision);
            if (rc) return rc;
            remap[ci] = nc++;
        }
        DevLeaf& d = a.leaves[L];
        d.comp = remap[ci];
        d.sigma = leaves[L].sigma;
        d.g0 = leaves[L].gamma[0]; d.g1 = leaves[L].gamma[1]; d.g2 = leaves[L].gamma[2];
        d.ampl = leaves[L].ampl;
        d.pad = 0;
    }
    a.n_leaves = n_leaves;
    // pairs of consecutive Multipole leaves that one walk can serve (pad = 1 on the
    // first): the same transform, radial grid, column structure and harmonic count
    for (int L = 0; L + 1 < n_leaves; ++L) {
        const DevLeaf& p = a.leaves[L];
        const DevLeaf& q = a.leaves[L + 1];
        const DevComp& c1 = a.comps[p.comp];
        const DevComp& c2 = a.comps[q.comp];
        if (c1.kind != AGB_KIND_MULTIPOLE || c2.kind != AGB_KIND_MULTIPOLE) continue;
        if (!(c1.structure == AGB_STRUCT_EVEN || c1.structure == AGB_STRUCT_ALL)) continue;
        if (c2.structure != c1.structure || c2.lmax != c1.lmax || c2.n_lm != c1.n_lm ||
            c2.n_int != c1.n_int || c2.p[0] != c1.p[0] || c2.p[1] != c1.p[1] ||
            c2.p[2] != c1.p[2] || c2.layout != c1.layout)
            continue;
        if (p.sigma != q.sigma || p.g0 != q.g0 || p.g1 != q.g1 || p.g2 != q.g2) continue;
        if (precision != AGB_PREC_MIXED || !c1.table32 || !c2.table32) continue;
        a.leaves[L].pad = 1;
        ++L;                      // a leaf belongs to at most one pair
    }
    (void)n_comps;
    return AGB_OK;
}

static std::atomic<unsigned long long> g_bin_attr_set{0};     // one bit per device

// Sort the points by interval into the workspace; sets a.xyz / a.perm.
// with_perm false: the caller needs no sorted position -> point map (outputs staged in
// sorted order and gathered through the keys, no per-point cotangents to read), so
// bin_scatter skips those 4-byte scattered writes and a.perm stays null
static int run_binning(EvalArgs& a, const BinPlan& b, const double* xyz, int64_t n, char* ws,
                       cudaStream_t st, bool with_perm = true)
{
    int* keys = (int*)ws;
    int* perm = (int*)(ws + al256(4 * (size_t)n));
    double* xs = (double*)(ws + 2 * al256(4 * (size_t)n));
    int* counts = (int*)(ws + 2 * al256(4 * (size_t)n) + al256(24 * (size_t)n));
    int* cursor = (int*)((char*)counts + al256(4 * (size_t)b.n_bins));
    const size_t smem1 = 4 * (size_t)b.n_bins, smem3 = 8 * (size_t)b.n_bins;
    const unsigned long long bit = 1ull << current_device();
    if (!(g_bin_attr_set.load(std::memory_order_acquire) & bit)) {
        // idempotent: two threads doing this at once set the same attributes
        cudaFuncSetAttribute(bin_count, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * AGB_MAX_BINS);
        cudaFuncSetAttribute(bin_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * AGB_MAX_BINS);
        g_bin_attr_set.fetch_or(bit, std::memory_order_release);
    }
    if (cudaMemsetAsync(counts, 0, 4 * (size_t)b.n_bins, st) != cudaSuccess)
        return set_err(AGB_ERR_DEVICE, "agb_eval: memset of bin counts failed");
    // points per block: the largest power of two from 512 to 4096 that still gives
    // every SM 4 blocks (each thread's atomics and loads are sequential, so small calls
    // need many blocks in flight; 0.5M points: 1024 blocks instead of 128)
    const long long per4 = n / ((long long)num_sms() * 4);
    int tile = 512;
    while (tile < AGB_BIN_TILE_MAX && 2LL * tile <= per4) tile <<= 1;
    const int tiles = (int)((n + tile - 1) / tile);
    bin_count<<<tiles, 256, smem1, st>>>(xyz, n, tile, b.key, b.n_bins, keys, counts);
    int rc = check_launch("bin_count");
    if (rc) return rc;
    bin_scan<<<1, 1024, 0, st>>>(counts, cursor, b.n_bins);
    if ((rc = check_launch("bin_scan"))) return rc;
    bin_scatter<<<tiles, 256, smem3, st>>>(xyz, n, tile, b.n_bins, keys, cursor,
                                           with_perm ? perm : nullptr, xs);
    if ((rc = check_launch("bin_scatter"))) return rc;
    a.xyz = xs;
    a.perm = with_perm ? perm : nullptr;
    return AGB_OK;
}

static thread_local const double* g_vjp_phi = nullptr;    // set by agb_eval_vjp for one call
static thread_local const double* g_vjp_force = nullptr;

static int eval_impl(const agb_component* comps, int n_comps, const agb_leaf* leaves, int n_leaves,
                     const double* xyz, int64_t n, int mode, int precision, double* phi,
                     double* grad, double* hess, double* rho, int out_flags, void* workspace,
                     size_t workspace_bytes, bool own_ws, void* stream, bool fixed_ws = false)
{
    int rc = validate(comps, n_comps, leaves, n_leaves, xyz, n, mode, precision, phi, grad, hess, rho);
    if (rc) return rc;
    if (((out_flags >> AGB_OUT_BLOCK_SHIFT) & 3) == 3)
        return set_err(AGB_ERR_ARG, "agb_eval: block-size code 3 in out_flags is not defined");
    if (n == 0) return AGB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    static thread_local EvalArgs a;
    memset(&a, 0, sizeof(a));
    a.n = n; a.out_flags = out_flags; a.soa = 0; a.xyz = xyz; a.perm = nullptr;
    a.phi = phi; a.grad = grad; a.hess = hess; a.rho = rho;
    a.gphi = g_vjp_phi; a.gforce = g_vjp_force;
    if ((rc = pack_args(a, comps, n_comps, leaves, n_leaves, precision))) return rc;

    const BinPlan b = plan_binning(comps, leaves, n_leaves, n, out_flags);
    // sorted-order output staging when the workspace has room for it (always for
    // agb_eval's own allocation and for workspaces sized by agb_eval_workspace_bytes)
    const size_t staged = ws_bytes_staged(b, n);
    const bool stage = b.on && (own_ws || (workspace && workspace_bytes >= staged));
    const size_t need = stage ? staged : ws_bytes(b, n);
    void* ws = workspace;
    if (need) {
        if (own_ws) {
            if (cudaMallocAsync(&ws, need, st) != cudaSuccess)
                return set_err(AGB_ERR_DEVICE, "agb_eval: cannot allocate %zu bytes of scratch", need);
        } else if (!ws || workspace_bytes < need) {
            if (fixed_ws)
                return set_err(AGB_ERR_UNSUPPORTED, "agb_eval_static: needs %zu bytes of scratch, "
                               "more than its fixed %zu (use agb_eval or agb_eval_ws)", need,
                               workspace_bytes);
            return set_err(AGB_ERR_ARG, "agb_eval_ws: workspace of %zu bytes is smaller than the "
                           "%zu bytes agb_eval_workspace_bytes asks for", workspace_bytes, need);
        }
        if ((uintptr_t)ws & 255u) {
            if (own_ws) cudaFreeAsync(ws, st);
            return set_err(AGB_ERR_ARG, "agb_eval_ws: workspace must be 256-byte aligned");
        }
        const bool vjp = mode == AGB_MODE_VJP || mode == AGB_MODE_VJPF;
        rc = run_binning(a, b, xyz, n, (char*)ws, st, !stage || vjp);
        if (stage) {
            a.stage = (double*)((char*)ws + ws_bytes(b, n));
            a.dest = (const int*)ws;             // bin_scatter leaves pos of point i in keys[i]
        }
    }
    if (!rc) rc = launch_mode(mode, precision, a, st);
    if (need && own_ws) cudaFreeAsync(ws, st);
    return rc;
}

extern "C" size_t agb_eval_workspace_bytes(const agb_component* comps, int n_comps,
                                           const agb_leaf* leaves, int n_leaves, int64_t n,
                                           int out_flags)
{
    if (!comps || !leaves || n_leaves < 1 || n_comps < 1) return 0;
    for (int L = 0; L < n_leaves; ++L)
        if (leaves[L].comp < 0 || leaves[L].comp >= n_comps) return 0;
    return ws_bytes_staged(plan_binning(comps, leaves, n_leaves, n, out_flags), n);
}

extern "C" int64_t agb_eval_wave_points(const agb_component* comps, int n_comps,
                                        const agb_leaf* leaves, int n_leaves, int mode,
                                        int precision)
{
    if (!comps || !leaves || n_leaves < 1 || n_comps < 1) return 0;
    bool an = true;
    for (int L = 0; L < n_leaves; ++L) {
        if (leaves[L].comp < 0 || leaves[L].comp >= n_comps) return 0;
        const int k = comps[leaves[L].comp].kind;
        if (k == AGB_KIND_MULTIPOLE || k == AGB_KIND_CYLSPLINE) an = false;
    }
    const bool mixed = precision == AGB_PREC_MIXED;
    switch (mode) {
    case AGB_MODE_POT:  return mixed ? eval_wave_points<AGB_MODE_POT, float>() : eval_wave_points<AGB_MODE_POT, double>();
    case AGB_MODE_GRAD: return mixed ? eval_wave_points<AGB_MODE_GRAD, float>() : eval_wave_points<AGB_MODE_GRAD, double>();
    case AGB_MODE_HESS: return mixed ? eval_wave_points<AGB_MODE_HESS, float>() : eval_wave_points<AGB_MODE_HESS, double>();
    case AGB_MODE_DENS: return mixed ? eval_wave_points<AGB_MODE_DENS, float>() : eval_wave_points<AGB_MODE_DENS, double>();
    case AGB_MODE_VJP:
        if (an) return eval_wave_points<AGB_MODE_VJP, double, true>();
        return mixed ? eval_wave_points<AGB_MODE_VJP, float>() : eval_wave_points<AGB_MODE_VJP, double>();
    default: return 0;
    }
}

extern "C" int agb_eval(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                        int n_leaves, const double* xyz, int64_t n, int mode, int precision,
                        double* phi, double* grad, double* hess, double* rho, int out_flags,
                        void* stream)
{
    return eval_impl(comps, n_comps, leaves, n_leaves, xyz, n, mode, precision, phi, grad, hess,
                     rho, out_flags, nullptr, 0, true, stream);
}

extern "C" int agb_eval_vjp(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                            int n_leaves, const double* xyz, int64_t n, int precision,
                            const double* g_phi, const double* g_force, double* g_xyz,
                            void* workspace, size_t workspace_bytes, void* stream)
{
    g_vjp_phi = g_phi;
    g_vjp_force = g_force;
    const int rc = eval_impl(comps, n_comps, leaves, n_leaves, xyz, n, AGB_MODE_VJP, precision,
                             nullptr, g_xyz, nullptr, nullptr, 0, workspace, workspace_bytes,
                             workspace == nullptr, stream);
    g_vjp_phi = nullptr;
    g_vjp_force = nullptr;
    return rc;
}

extern "C" int agb_eval_vjp_force(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                                  int n_leaves, const double* xyz, int64_t n, int precision,
                                  const double* g_phi, const double* g_force, double* g_xyz,
                                  double* force, void* workspace, size_t workspace_bytes,
                                  void* stream)
{
    g_vjp_phi = g_phi;
    g_vjp_force = g_force;
    const int rc = eval_impl(comps, n_comps, leaves, n_leaves, xyz, n, AGB_MODE_VJPF, precision,
                             nullptr, g_xyz, force, nullptr, 0, workspace, workspace_bytes,
                             workspace == nullptr, stream);
    g_vjp_phi = nullptr;
    g_vjp_force = nullptr;
    return rc;
}

extern "C" int agb_eval_ws(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                           int n_leaves, const double* xyz, int64_t n, int mode, int precision,
                           double* phi, double* grad, double* hess, double* rho, int out_flags,
                           void* workspace, size_t workspace_bytes, void* stream)
{
    return eval_impl(comps, n_comps, leaves, n_leaves, xyz, n, mode, precision, phi, grad, hess,
                     rho, out_flags, workspace, workspace_bytes, false, stream);
}

// ---------------------------------------------------------------------------
// time plans: leaves computed on the device from a device-resident step
// ---------------------------------------------------------------------------
struct agb_time_plan {
    int n;
    int device;
    agb_leaf_prog progs[AGB_MAX_LEAVES];
    int max_comp[AGB_MAX_LEAVES];     // largest component index a program can pick
    int evo_lo[AGB_MAX_LEAVES];       // EVOLVE: first snapshot component (else comp)
    double* table_dev;
    double* table_host;
    int64_t n_table;
};

static bool tp_increasing(const double* x, int n)
{
    for (int i = 1; i < n; ++i)
        if (!(x[i] > x[i - 1])) return false;
    return true;
}

// size in doubles of an op's data block (0: malformed), checked against the table
static int64_t tp_op_size(int op, const double* d, int64_t avail)
{
    if (avail < 1) return 0;
    if (op == AGB_OP_SHIFT) {
        if (d[0] == 0.0) return avail >= 4 ? 4 : 0;
        if (d[0] != 1.0 || avail < 16) return 0;
        const double T = d[1];
        if (!(T >= 2.0 && T <= 1.0e7) || T != (double)(int64_t)T) return 0;
        const int64_t need = 16 + (int64_t)T + 12 * ((int64_t)T - 1);
        if (need > avail || !tp_increasing(d + 16, (int)T)) return 0;
        return need;
    }
    if (op == AGB_OP_SCALE) {
        if (d[0] == 0.0) return (avail >= 3 && d[1] != 0.0) ? 3 : 0;
        if (d[0] != 1.0 || avail < 14) return 0;
        const double T = d[1];
        if (!(T >= 2.0 && T <= 1.0e7) || T != (double)(int64_t)T) return 0;
        if (d[8] != 0.0 && d[8] != 1.0) return 0;
        const int64_t need = 14 + (int64_t)T + 4 * ((int64_t)T - 1) * (d[8] != 0.0 ? 2 : 1);
        if (need > avail || !tp_increasing(d + 14, (int)T)) return 0;
        return need;
    }
    if (op == AGB_OP_EVOLVE) {
        if (avail < 3) return 0;
        const double n = d[0];
        if (!(n >= 1.0 && n <= 1.0e6) || n != (double)(int64_t)n) return 0;
        if (d[1] != 0.0 && d[1] != 1.0) return 0;
        const int64_t need = 2 + (int64_t)n;
        if (need > avail || !tp_increasing(d + 2, (int)n)) return 0;
        return need;
    }
    return 0;
}

extern "C" int agb_time_plan_create(const agb_leaf_prog* progs, int n_progs, const double* table,
                                    int64_t n_table, agb_time_plan** out)
{
    if (!out) return set_err(AGB_ERR_ARG, "agb_time_plan_create: out is null");
    *out = nullptr;
    if (!progs || n_progs < 1 || n_progs > AGB_MAX_LEAVES)
        return set_err(AGB_ERR_ARG, "agb_time_plan_create: %d programs (1..%d)", n_progs, AGB_MAX_LEAVES);
    if (n_table < 0 || (n_table > 0 && !table))
        return set_err(AGB_ERR_ARG, "agb_time_plan_create: bad table");
    agb_time_plan* p = (agb_time_plan*)calloc(1, sizeof(agb_time_plan));
    if (!p) return set_err(AGB_ERR_DEVICE, "agb_time_plan_create: out of host memory");
    p->n = n_progs;
    for (int i = 0; i < n_progs; ++i) {
        const agb_leaf_prog& g = progs[i];
        int evolves = 0, maxc = g.comp;
        if (g.comp < 0 || g.n_ops < 0 || g.n_ops > AGB_MAX_LEAF_OPS || g.slot < 0 || g.slot > 1) {
            free(p);
            return set_err(AGB_ERR_ARG, "agb_time_plan_create: program %d: bad comp, op count or slot", i);
        }
        for (int k = 0; k < g.n_ops; ++k) {
            const int64_t at = g.arg[k];
            const int64_t sz = (at >= 0 && at < n_table) ? tp_op_size(g.op[k], table + at, n_table - at) : 0;
            if (sz == 0) {
                free(p);
                return set_err(AGB_ERR_ARG, "agb_time_plan_create: program %d op %d (kind %d) has "
                               "malformed table data at %lld", i, k, g.op[k], (long long)at);
            }
            if (g.op[k] == AGB_OP_EVOLVE) {
                const int n = (int)table[at];
                const bool interp = table[at + 1] != 0.0;
                if (++evolves > 1 || (g.slot == 1 && (!interp || n < 2))) {
                    free(p);
                    return set_err(AGB_ERR_ARG, "agb_time_plan_create: program %d: one EVOLVE op "
                                   "at most, slot 1 needs interpolation of >= 2 snapshots", i);
                }
                maxc = g.comp + n - 1;
            }
        }
        p->progs[i] = g;
        p->progs[i].pair = 0;           // decided per call (agb_eval_timed)
        p->max_comp[i] = maxc;
    }
    p->n_table = n_table;
    const size_t bytes = sizeof(double) * (size_t)(n_table > 0 ? n_table : 1);
    p->table_host = (double*)malloc(bytes);
    if (!p->table_host) {
        free(p);
        return set_err(AGB_ERR_DEVICE, "agb_time_plan_create: out of host memory");
    }
    if (n_table > 0) memcpy(p->table_host, table, bytes);
    // without any CUDA device the plan serves agb_time_plan_leaves_host only
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev < 1) {
        cudaGetLastError();
        p->device = -1;
        *out = p;
        return AGB_OK;
    }
    cudaGetDevice(&p->device);
    if (cudaMalloc(&p->table_dev, bytes) != cudaSuccess) {
        free(p->table_host);
        free(p);
        return set_err(AGB_ERR_DEVICE, "agb_time_plan_create: cannot allocate %zu bytes", bytes);
    }
    if (n_table > 0) {
        if (cudaMemcpy(p->table_dev, table, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(p->table_dev);
            free(p->table_host);
            free(p);
            return set_err(AGB_ERR_DEVICE, "agb_time_plan_create: upload of the table failed");
        }
    }
    *out = p;
    return AGB_OK;
}

extern "C" void agb_time_plan_destroy(agb_time_plan* p)
{
    if (!p) return;
    if (p->table_dev) {
        int cur = 0;
        cudaGetDevice(&cur);
        if (cur != p->device) cudaSetDevice(p->device);
        cudaFree(p->table_dev);
        if (cur != p->device) cudaSetDevice(cur);
    }
    free(p->table_host);
    free(p);
}

extern "C" int agb_time_plan_leaves_host(const agb_time_plan* p, double t, agb_leaf* leaves)
{
    if (!p || !leaves) return set_err(AGB_ERR_ARG, "agb_time_plan_leaves_host: null argument");
    for (int i = 0; i < p->n; ++i) {
        DevLeaf o;
        tp_leaf(p->progs[i], p->table_host, t, o);
        leaves[i].comp = o.comp;
        leaves[i].reserved = 0;
        leaves[i].sigma = o.sigma;
        leaves[i].gamma[0] = o.g0; leaves[i].gamma[1] = o.g1; leaves[i].gamma[2] = o.g2;
        leaves[i].ampl = o.ampl;
    }
    return AGB_OK;
}

static int launch_time_leaves(const agb_time_plan* p, const int* pair, const int64_t* step,
                              double t0, double dt, double off, DevLeaf* out, cudaStream_t st)
{
    static thread_local TimeLeafArgs ta;
    memset(&ta, 0, sizeof(ta));
    ta.n = p->n;
    for (int i = 0; i < p->n; ++i) {
        ta.progs[i] = p->progs[i];
        ta.progs[i].pair = pair ? pair[i] : 0;
    }
    ta.table = p->table_dev;
    ta.step = (const long long*)step;
    ta.t0 = t0; ta.dt = dt; ta.off = off;
    ta.out = out;
    time_leaves_kernel<<<1, 32, 0, st>>>(ta);
    return check_launch("time_leaves_kernel");
}

extern "C" int agb_time_plan_leaves(const agb_time_plan* p, const int64_t* step, double t0,
                                    double dt, double off, agb_leaf* leaves_dev, void* stream)
{
    if (!p || !leaves_dev) return set_err(AGB_ERR_ARG, "agb_time_plan_leaves: null argument");
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->device)
        return set_err(AGB_ERR_ARG, "agb_time_plan_leaves: plan lives on device %d, current is %d",
                       p->device, cur);
    static_assert(sizeof(agb_leaf) == sizeof(DevLeaf), "agb_leaf and DevLeaf must share a layout");
    return launch_time_leaves(p, nullptr, step, t0, dt, off, (DevLeaf*)leaves_dev,
                              (cudaStream_t)stream);
}

// The component a program uses at any time, as a static leaf (for validation and
// for choosing the sort key: an EVOLVE program stands for its first snapshot).
static void tp_template_leaves(const agb_time_plan* p, agb_leaf* lv)
{
    for (int i = 0; i < p->n; ++i) {
        memset(&lv[i], 0, sizeof(agb_leaf));
        lv[i].comp = p->progs[i].comp;
        lv[i].sigma = 1.0;
        lv[i].ampl = 1.0;
    }
}

static bool tp_same_ops(const agb_leaf_prog& a, const agb_leaf_prog& b)
{
    if (a.n_ops != b.n_ops || a.comp != b.comp) return false;
    for (int k = 0; k < a.n_ops; ++k)
        if (a.op[k] != b.op[k] || a.arg[k] != b.arg[k]) return false;
    return true;
}

// one harmonic walk may serve programs L and L+1 (the two slots of one Evolving):
// the same modifier chain, and every snapshot a Multipole of one grid and column
// structure with an FP32 table
static void tp_pairs(const agb_time_plan* p, const agb_component* comps, int precision, int* pair)
{
    for (int i = 0; i < p->n; ++i) pair[i] = 0;
    if (precision != AGB_PREC_MIXED) return;
    for (int L = 0; L + 1 < p->n; ++L) {
        const agb_leaf_prog& a = p->progs[L];
        const agb_leaf_prog& b = p->progs[L + 1];
        if (!tp_same_ops(a, b) || a.slot != 0 || b.slot != 1 || p->max_comp[L] == a.comp) continue;
        const agb_component& c0 = comps[a.comp];
        bool ok = c0.kind == AGB_KIND_MULTIPOLE &&
                  (c0.structure == AGB_STRUCT_EVEN || c0.structure == AGB_STRUCT_ALL);
        for (int c = a.comp + 1; ok && c <= p->max_comp[L]; ++c) {
            const agb_component& q = comps[c];
            ok = q.kind == AGB_KIND_MULTIPOLE && q.structure == c0.structure &&
                 q.lmax == c0.lmax && q.n_lm == c0.n_lm && q.n_int == c0.n_int &&
                 q.layout == c0.layout && q.p[0] == c0.p[0] && q.p[1] == c0.p[1] &&
                 q.p[2] == c0.p[2] && q.table32 != nullptr;
        }
        ok = ok && c0.table32 != nullptr;
        if (ok) {
            pair[L] = 1;
            ++L;
        }
    }
}

static const size_t TP_LEAF_BYTES = 256 * ((sizeof(DevLeaf) * AGB_MAX_LEAVES + 255) / 256);

extern "C" size_t agb_eval_timed_workspace_bytes(const agb_component* comps, int n_comps,
                                                 const agb_time_plan* p, int64_t n, int out_flags)
{
    if (!comps || !p || n_comps < 1) return 0;
    for (int i = 0; i < p->n; ++i)
        if (p->max_comp[i] >= n_comps) return 0;
    agb_leaf lv[AGB_MAX_LEAVES];
    tp_template_leaves(p, lv);
    return TP_LEAF_BYTES + ws_bytes_staged(plan_binning(comps, lv, p->n, n, out_flags), n);
}

extern "C" int agb_eval_timed(const agb_component* comps, int n_comps, const agb_time_plan* p,
                              const int64_t* step, double t0, double dt, double off,
                              const double* xyz, int64_t n, int mode, int precision, double* phi,
                              double* grad, double* hess, double* rho, int out_flags,
                              void* workspace, size_t workspace_bytes, void* stream)
{
    if (!p) return set_err(AGB_ERR_ARG, "agb_eval_timed: plan is null");
    if (mode != AGB_MODE_POT && mode != AGB_MODE_GRAD && mode != AGB_MODE_HESS &&
        mode != AGB_MODE_DENS)
        return set_err(AGB_ERR_ARG, "agb_eval_timed: mode %d is not supported", mode);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->device)
        return set_err(AGB_ERR_ARG, "agb_eval_timed: plan lives on device %d, current is %d",
                       p->device, cur);
    for (int i = 0; i < p->n; ++i)
        if (p->max_comp[i] >= n_comps)
            return set_err(AGB_ERR_ARG, "agb_eval_timed: program %d uses component %d of %d", i,
                           p->max_comp[i], n_comps);
    if (n_comps > AGB_MAX_COMPONENTS)
        return set_err(AGB_ERR_UNSUPPORTED, "agb_eval_timed: more than %d components",
                       AGB_MAX_COMPONENTS);
    agb_leaf lv[AGB_MAX_LEAVES];
    tp_template_leaves(p, lv);
    int rc = validate(comps, n_comps, lv, p->n, xyz, n, mode, precision, phi, grad, hess, rho);
    if (rc) return rc;
    if (n == 0) return AGB_OK;
    if (!workspace || ((uintptr_t)workspace & 255u) || workspace_bytes < TP_LEAF_BYTES)
        return set_err(AGB_ERR_ARG, "agb_eval_timed: workspace of at least "
                       "agb_eval_timed_workspace_bytes() bytes, 256-byte aligned, is required");
    cudaStream_t st = (cudaStream_t)stream;
    static thread_local EvalArgs a;
    memset(&a, 0, sizeof(a));
    a.n = n; a.out_flags = out_flags; a.soa = 0; a.xyz = xyz; a.perm = nullptr;
    a.phi = phi; a.grad = grad; a.hess = hess; a.rho = rho;
    for (int c = 0; c < n_comps; ++c)
        if ((rc = comp_to_dev(comps[c], a.comps[c], precision))) return rc;
    a.n_leaves = p->n;
    DevLeaf* dl = (DevLeaf*)workspace;
    a.dleaves = dl;
    int pair[AGB_MAX_LEAVES];
    tp_pairs(p, comps, precision, pair);
    if ((rc = launch_time_leaves(p, pair, step, t0, dt, off, dl, st))) return rc;
    char* ws = (char*)workspace + TP_LEAF_BYTES;
    const size_t room = workspace_bytes - TP_LEAF_BYTES;
    BinPlan b = plan_binning(comps, lv, p->n, n, out_flags);
    if (b.on) {
        b.key.leaf = dl + b.leaf;
        const size_t staged = ws_bytes_staged(b, n);
        const size_t need = ws_bytes(b, n);
        if (room < need)
            return set_err(AGB_ERR_ARG, "agb_eval_timed: workspace of %zu bytes is smaller than "
                           "the %zu bytes agb_eval_timed_workspace_bytes asks for",
                           workspace_bytes, need + TP_LEAF_BYTES);
        const bool stage = room >= staged;
        const bool vjp = mode == AGB_MODE_VJP || mode == AGB_MODE_VJPF;
        if ((rc = run_binning(a, b, xyz, n, ws, st, !stage || vjp))) return rc;
        if (stage) {
            a.stage = (double*)(ws + ws_bytes(b, n));
            a.dest = (const int*)ws;
        }
    }
    return launch_mode(mode, precision, a, st);
}

extern "C" int agb_leapfrog_kick_drift(double* x, double* v, const double* F, int64_t n,
                                       double h1, double h2, double dt, int flags, int64_t* step,
                                       void* stream)
{
    if (n < 0) return set_err(AGB_ERR_ARG, "agb_leapfrog_kick_drift: negative count");
    if (flags & ~15) return set_err(AGB_ERR_ARG, "agb_leapfrog_kick_drift: unknown flags %d", flags);
    if ((flags & 8) && !step) return set_err(AGB_ERR_ARG, "agb_leapfrog_kick_drift: step is null");
    if (n == 0 && !(flags & 8)) return AGB_OK;
    if (n > 0 && (!x || !v || !F)) return set_err(AGB_ERR_ARG, "agb_leapfrog_kick_drift: null array");
    const long long m = 3LL * n;
    kick_drift_kernel<<<grid_for(m > 0 ? m : 1), 256, 0, (cudaStream_t)stream>>>(
        x, v, F, m, h1, h2, dt, flags, (long long*)step);
    return check_launch("kick_drift_kernel");
}

// ---------------------------------------------------------------------------
// gradient w.r.t. one Multipole leaf's quintic coefficients
// ---------------------------------------------------------------------------
extern "C" size_t agb_multipole_adjoint_workspace_bytes(const agb_component* comp,
                                                        const agb_leaf* leaf, int64_t n,
                                                        int with_force)
{
    if (!comp || !leaf) return 0;
    agb_leaf l = *leaf;
    l.comp = 0;
    const BinPlan b = plan_binning(comp, &l, 1, n, 0);
    if (!b.on) return 0;
    return ws_bytes(b, n) + al256(8 * (size_t)(with_force ? 6 : 3) * (size_t)n);
}

extern "C" size_t agb_multipole_table_vjp_workspace_bytes(const agb_component* comp,
                                                          const agb_leaf* leaf, int64_t n)
{
    if (!comp || !leaf) return 0;
    agb_leaf l = *leaf;
    l.comp = 0;
    return ws_bytes(plan_binning(comp, &l, 1, n, 0), n);
}

extern "C" int agb_multipole_table_vjp(const agb_component* comp, const agb_leaf* leaf,
                                       const double* xyz, int64_t n, const double* g_phi,
                                       const double* g_force, double* g_table, double* g_const,
                                       void* workspace, size_t workspace_bytes, void* stream)
{
    if (!comp || !leaf || !g_table) return set_err(AGB_ERR_ARG, "agb_multipole_table_vjp: null argument");
    if (comp->kind != AGB_KIND_MULTIPOLE)
        return set_err(AGB_ERR_ARG, "agb_multipole_table_vjp: component is not a Multipole");
    if (comp->layout != AGB_LAYOUT_INTERVAL_MAJOR)
        return set_err(AGB_ERR_ARG, "agb_multipole_table_vjp: the table must be interval-major");
    if (n < 0) return set_err(AGB_ERR_ARG, "agb_multipole_table_vjp: negative point count");
    if (n == 0) return AGB_OK;
    if (!xyz) return set_err(AGB_ERR_ARG, "agb_multipole_table_vjp: xyz is null");
    static thread_local MPGradArgs g;
    memset(&g, 0, sizeof(g));
    int rc = comp_to_dev(*comp, g.c, AGB_PREC_FP64);
    if (rc) return rc;
    g.leaf.comp = 0; g.leaf.sigma = leaf->sigma; g.leaf.ampl = leaf->ampl;
    g.leaf.g0 = leaf->gamma[0]; g.leaf.g1 = leaf->gamma[1]; g.leaf.g2 = leaf->gamma[2];
    g.n = n; g.xyz = xyz; g.perm = nullptr; g.gphi = g_phi; g.gforce = g_force; g.grad = g_table;
    g.gconst = g_const;
    cudaStream_t st = (cudaStream_t)stream;
    agb_leaf l = *leaf;
    l.comp = 0;
    const BinPlan b = plan_binning(comp, &l, 1, n, 0);
    const size_t need = ws_bytes(b, n);
    void* ws = workspace;
    const bool own = (workspace == nullptr);
    if (need) {
        if (own) {
            if (cudaMallocAsync(&ws, need, st) != cudaSuccess)
                return set_err(AGB_ERR_DEVICE, "agb_multipole_table_vjp: cannot allocate scratch");
        } else if (workspace_bytes < need || ((uintptr_t)ws & 255u)) {
            return set_err(AGB_ERR_ARG, "agb_multipole_table_vjp: workspace too small or misaligned");
        }
        static thread_local EvalArgs tmp;
        memset(&tmp, 0, sizeof(tmp));
        rc = run_binning(tmp, b, xyz, n, (char*)ws, st);
        g.xyz = tmp.xyz;
        g.perm = tmp.perm;
    }
    if (!rc) {
        mp_grad_kernel<<<grid_for(n), 256, 0, st>>>(g);
        rc = check_launch("mp_grad_kernel");
    }
    if (need && own) cudaFreeAsync(ws, st);
    return rc;
}

// ---------------------------------------------------------------------------
// fused adjoint of one Multipole leaf (position VJP + coefficient gradient)
// ---------------------------------------------------------------------------
// keep: (agb_adjoint_step) the per-point results stay staged in the workspace, in
// sorted order, with the sorted position of point i in dest[i]; they are not added
// to g_xyz / force (which may then be null; with_force sets the record size)
struct AdjKeep {
    bool on;
    bool with_force;
    const int* dest;
    const double* stage;
};

static int multipole_adjoint_impl(const agb_component* comp, const agb_leaf* leaf,
                                  const double* xyz, int64_t n, int precision,
                                  const double* g_phi, const double* g_force, double* g_xyz,
                                  double* force, double* g_table, double* g_const,
                                  void* workspace, size_t workspace_bytes, void* stream,
                                  AdjKeep* keep = nullptr, double g_force_scale = 1.0)
{
    const bool keep_on = keep && keep->on;
    if (!comp || !leaf || !g_table || (!g_xyz && !keep_on))
        return set_err(AGB_ERR_ARG, "agb_multipole_adjoint: null argument");
    if (comp->kind != AGB_KIND_MULTIPOLE || comp->layout != AGB_LAYOUT_INTERVAL_MAJOR ||
        comp->structure == AGB_STRUCT_LIST)
        return set_err(AGB_ERR_ARG, "agb_multipole_adjoint: needs an interval-major Multipole "
                       "table with a regular column structure");
    if (precision != AGB_PREC_FP64 && precision != AGB_PREC_MIXED)
        return set_err(AGB_ERR_ARG, "agb_multipole_adjoint: unknown precision %d", precision);
    if (n < 0) return set_err(AGB_ERR_ARG, "agb_multipole_adjoint: negative point count");
    if (n == 0) return AGB_OK;
    if (!xyz) return set_err(AGB_ERR_ARG, "agb_multipole_adjoint: xyz is null");
    static thread_local MPAdjArgs g;
    memset(&g, 0, sizeof(g));
    int rc = comp_to_dev(*comp, g.c, precision);
    if (rc) return rc;
    g.leaf.comp = 0; g.leaf.sigma = leaf->sigma; g.leaf.ampl = leaf->ampl;
    g.leaf.g0 = leaf->gamma[0]; g.leaf.g1 = leaf->gamma[1]; g.leaf.g2 = leaf->gamma[2];
    g.n = n; g.xyz = xyz; g.perm = nullptr; g.gphi = g_phi; g.gforce = g_force;
    g.gx = g_xyz; g.grad = g_table; g.force = force; g.gconst = g_const;
    g.gforce_scale = g_force_scale;
    cudaStream_t st = (cudaStream_t)stream;
    agb_leaf l = *leaf;
    l.comp = 0;
    const BinPlan b = plan_binning(comp, &l, 1, n, keep_on ? AGB_OUT_BIN_ALWAYS : 0);
    const size_t rec = (force || (keep_on && keep->with_force)) ? 6 : 3;
    const size_t staged = b.on ? ws_bytes(b, n) + al256(8 * rec * (size_t)n) : 0;
    const bool own = (workspace == nullptr);
    // with room for them, the per-point results are written in sorted order and added
    // back in input order by adj_unpermute_add (always for the library's own scratch)
    const bool stage = b.on && (own || workspace_bytes >= staged);
    if (keep_on && (!stage || own))
        return set_err(AGB_ERR_ARG, "agb_adjoint_step: a workspace of "
                       "agb_adjoint_step_workspace_bytes() bytes is required");
    g.stage_rec = (int)rec;
    const size_t need = stage ? staged : ws_bytes(b, n);
    void* ws = workspace;
    if (need) {
        if (own) {
            if (cudaMallocAsync(&ws, need, st) != cudaSuccess)
                return set_err(AGB_ERR_DEVICE, "agb_multipole_adjoint: cannot allocate scratch");
        } else if (workspace_bytes < need || ((uintptr_t)ws & 255u)) {
            return set_err(AGB_ERR_ARG, "agb_multipole_adjoint: workspace too small or misaligned");
        }
        static thread_local EvalArgs tmp;
        memset(&tmp, 0, sizeof(tmp));
        rc = run_binning(tmp, b, xyz, n, (char*)ws, st);
        g.xyz = tmp.xyz;
        g.perm = tmp.perm;
        if (stage) g.stage = (double*)((char*)ws + ws_bytes(b, n));
    }
    if (!rc) {
        // per warp: the (U, V) tile, plus the interval accumulator.  Blocks of 2 warps
        // (64 threads at 255 registers, 4 resident per SM: the same 8 warps as one block
        // of 256, scheduled in finer pieces), four waves of them: the backward leapfrog
        // step at 2.1M particles 2.006 -> 1.925 ms (two waves 1.955, one 1.945, eight
        // 1.984 ms; 128-thread blocks 1.968, 32-thread 1.986 ms in two waves).
        // 384 threads at 168 registers spilled and made the step 22 % slower.
        const int grid = (int)std::min<long long>((long long)num_sms() * 16, (n + 63) / 64);
        const long long warps = (long long)grid * 2, groups = (n + 31) / 32;
        g.chunk = ((groups + warps - 1) / warps) * 32;
        const int tile = precision == AGB_PREC_MIXED ? adj_tile_bytes<float>() : adj_tile_bytes<double>();
        const size_t acc = (size_t)g.c.n_lm * 6 * sizeof(double);
        int optin = 0;
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                   current_device()) != cudaSuccess)
            optin = 48 * 1024;
        // + 64 bytes per warp: its sums of the builder-scalar gradients (g_const)
        const size_t cst = g_const ? 64 : 0;
        // staged when the SM holds the accumulators of all 8 warps of its 4 blocks
        g.staged = (size_t)8 * (tile + acc + cst) <= (size_t)optin;
        g.warp_smem = (int)((g.staged ? tile + acc : tile) + cst);
        const size_t smem = (size_t)2 * g.warp_smem;
        const void* fn = precision == AGB_PREC_MIXED ? (const void*)mp_adjoint_kernel<float>
                                                     : (const void*)mp_adjoint_kernel<double>;
        if (smem > (size_t)optin)
            rc = set_err(AGB_ERR_UNSUPPORTED, "agb_multipole_adjoint: needs %zu bytes of shared "
                         "memory per block, more than %d", smem, optin);
        else if (smem > 48 * 1024 &&
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            rc = set_err(AGB_ERR_DEVICE, "agb_multipole_adjoint: cannot reserve %zu bytes of shared "
                         "memory", smem);
        if (!rc) {
            if (precision == AGB_PREC_MIXED) mp_adjoint_kernel<float><<<grid, 64, smem, st>>>(g);
            else mp_adjoint_kernel<double><<<grid, 64, smem, st>>>(g);
            rc = check_launch("mp_adjoint_kernel");
        }
        if (!rc && g.stage && keep_on) {
            keep->dest = (const int*)ws;           // bin_scatter leaves pos of point i in keys[i]
            keep->stage = g.stage;
        } else if (!rc && g.stage) {
            const int* dest = (const int*)ws;       // bin_scatter leaves pos of point i in keys[i]
            if (force) adj_unpermute_add<6><<<grid_for(n), 256, 0, st>>>(dest, g.stage, n, g_xyz, force);
            else adj_unpermute_add<3><<<grid_for(n), 256, 0, st>>>(dest, g.stage, n, g_xyz, nullptr);
            rc = check_launch("adj_unpermute_add");
        }
    }
    if (need && own) cudaFreeAsync(ws, st);
    return rc;
}

// ---------------------------------------------------------------------------
// one backward step of the leapfrog adjoint in two launches: the fused
// Multipole adjoint (staged in sorted order), then per particle the analytic
// leaves' VJP and force at x, the staged Multipole part added, the adjoint
// kick and (DRIFT) the time-reversed drift -- the work of the analytic VJP
// launch, adj_unpermute_add, adjoint_kick_kernel and reverse_drift_kernel, with
// the same arithmetic in the same order
// ---------------------------------------------------------------------------
struct AdjStepPtrs {
    double* x;           // [N,3] positions at the VJP (reverse-drifted in place)
    double* vh;          // [N,3] half-step velocities (DRIFT)
    double* lx;          // [N,3] adjoint of x
    double* lv;          // [N,3] adjoint of v
    double* gF;          // [N,3] in: cotangent of F at x; out: c lv (unless lv_cot)
    const int* dest;     // sorted position of point i
    const double* stage; // [pos][stage_rec] Multipole VJP (and force)
    long long n;
    int stage_rec;
    int drift;
    int lv_cot;          // the cotangent of F is c_in lv (lv on entry); gF unused
    double dt, c, c_in, k, dt_drift;
};

// One thread per particle.  The staged record (read through its sorted
// position) and lv are loaded before the analytic leaves' arithmetic, so the
// latency of that gather overlaps the FP64 Hessian instead of following it.
__global__ void __launch_bounds__(64, 8)
adjoint_step_kernel(const __grid_constant__ EvalArgs a, const __grid_constant__ AdjStepPtrs p)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride) {
        const double* t = p.stage + (long long)p.stage_rec * __ldg(p.dest + i);
        const double x = p.x[3 * i], y = p.x[3 * i + 1], z = p.x[3 * i + 2];
        double lv0[3], tv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        #pragma unroll
        for (int q = 0; q < 3; ++q) {
            lv0[q] = p.lv[3 * i + q];
            tv[q] = __ldg(t + q);
        }
        if (p.drift) {
            #pragma unroll
            for (int q = 0; q < 3; ++q) tv[3 + q] = __ldg(t + 3 + q);
        }
        double f0, f1, f2;
        if (p.lv_cot) {
            f0 = p.c_in * lv0[0]; f1 = p.c_in * lv0[1]; f2 = p.c_in * lv0[2];
        } else {
            f0 = p.gF[3 * i]; f1 = p.gF[3 * i + 1]; f2 = p.gF[3 * i + 2];
        }
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
        double h[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int L = 0; L < a.n_leaves; ++L) {
            const DevLeaf& lf = a.leaves[L];
            if (lf.ampl == 0.0) continue;
            PointOut o;
            o.phi = 0.0; o.rho = 0.0;
            o.g[0] = o.g[1] = o.g[2] = 0.0;
            #pragma unroll
            for (int q = 0; q < 6; ++q) o.h[q] = 0.0;
            eval_component<AGB_MODE_HESS, double, true, true>(
                a.comps[lf.comp], lf.sigma * x - lf.g0, lf.sigma * y - lf.g1, lf.sigma * z - lf.g2, o);
            const double As = lf.ampl * lf.sigma, As2 = As * lf.sigma;
            g0 += As * o.g[0]; g1 += As * o.g[1]; g2 += As * o.g[2];
            #pragma unroll
            for (int q = 0; q < 6; ++q) h[q] += As2 * o.h[q];
        }
        // the analytic leaves' VJP (no potential cotangent) and force, as the VJP-force
        // mode of agb_eval_kernel writes them, then the Multipole part added
        double gx[3], F[3];
        gx[0] = 0.0 * g0 - (h[0] * f0 + h[3] * f1 + h[5] * f2);
        gx[1] = 0.0 * g1 - (h[3] * f0 + h[1] * f1 + h[4] * f2);
        gx[2] = 0.0 * g2 - (h[5] * f0 + h[4] * f1 + h[2] * f2);
        gx[0] += tv[0]; gx[1] += tv[1]; gx[2] += tv[2];
        if (p.drift) {
            F[0] = -g0 + tv[3]; F[1] = -g1 + tv[4]; F[2] = -g2 + tv[5];
        }
        const double pos[3] = {x, y, z};
        #pragma unroll
        for (int q = 0; q < 3; ++q) {
            const long long j = 3 * i + q;
            const double lxq = p.lx[j] + gx[q];
            const double lvq = fma(p.dt, lxq, lv0[q]);
            p.lx[j] = lxq;
            p.lv[j] = lvq;
            if (!p.lv_cot) p.gF[j] = p.c * lvq;
            if (p.drift) {
                const double v = fma(-p.k, F[q], p.vh[j]);
                p.vh[j] = v;
                p.x[j] = fma(-p.dt_drift, v, pos[q]);
            }
        }
    }
}

static int adjoint_step_check(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                              int n_leaves, int mp_leaf)
{
    if (!comps || !leaves || n_comps < 1 || n_leaves < 1 || mp_leaf < 0 || mp_leaf >= n_leaves)
        return set_err(AGB_ERR_ARG, "agb_adjoint_step: bad component or leaf list");
    if (n_leaves > AGB_MAX_LEAVES)
        return set_err(AGB_ERR_UNSUPPORTED, "agb_adjoint_step: %d leaves exceed %d", n_leaves,
                       AGB_MAX_LEAVES);
    for (int L = 0; L < n_leaves; ++L) {
        if (leaves[L].comp < 0 || leaves[L].comp >= n_comps)
            return set_err(AGB_ERR_ARG, "agb_adjoint_step: leaf %d refers to component %d of %d",
                           L, leaves[L].comp, n_comps);
        const int kind = comps[leaves[L].comp].kind;
        if (L == mp_leaf) {
            if (kind != AGB_KIND_MULTIPOLE)
                return set_err(AGB_ERR_ARG, "agb_adjoint_step: leaf %d is not a Multipole", L);
        } else if (kind == AGB_KIND_MULTIPOLE || kind == AGB_KIND_CYLSPLINE) {
            return set_err(AGB_ERR_UNSUPPORTED, "agb_adjoint_step: leaves other than the "
                           "Multipole must be analytic");
        }
    }
    return AGB_OK;
}

extern "C" size_t agb_adjoint_step_workspace_bytes(const agb_component* comps, int n_comps,
                                                   const agb_leaf* leaves, int n_leaves,
                                                   int mp_leaf, int64_t n, int flags)
{
    if (adjoint_step_check(comps, n_comps, leaves, n_leaves, mp_leaf)) return 0;
    agb_leaf l = leaves[mp_leaf];
    l.comp = 0;
    const BinPlan b = plan_binning(&comps[leaves[mp_leaf].comp], &l, 1, n, AGB_OUT_BIN_ALWAYS);
    if (!b.on) return 0;
    return ws_bytes(b, n) + al256(8 * (size_t)((flags & AGB_ADJ_DRIFT) ? 6 : 3) * (size_t)n);
}

extern "C" int agb_adjoint_step(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                                int n_leaves, int mp_leaf, int precision, double* x, double* vh,
                                double* lx, double* lv, double* gF, double* g_table,
                                double* g_const, int64_t n, double dt, double c, double c_in,
                                double k, double dt_drift, int flags, void* workspace,
                                size_t workspace_bytes, void* stream)
{
    int rc = adjoint_step_check(comps, n_comps, leaves, n_leaves, mp_leaf);
    if (rc) return rc;
    if (n < 0) return set_err(AGB_ERR_ARG, "agb_adjoint_step: negative count");
    if (n == 0) return AGB_OK;
    const bool drift = (flags & AGB_ADJ_DRIFT) != 0;
    const bool lv_cot = (flags & AGB_ADJ_LV_COT) != 0;
    if (!x || !lx || !lv || (!gF && !lv_cot) || !g_table || (drift && !vh))
        return set_err(AGB_ERR_ARG, "agb_adjoint_step: null array");
    AdjKeep keep;
    keep.on = true;
    keep.with_force = drift;
    keep.dest = nullptr;
    keep.stage = nullptr;
    rc = multipole_adjoint_impl(&comps[leaves[mp_leaf].comp], &leaves[mp_leaf], x, n, precision,
                                nullptr, lv_cot ? lv : gF, nullptr, nullptr, g_table, g_const,
                                workspace, workspace_bytes, stream, &keep,
                                lv_cot ? c_in : 1.0);
    if (rc) return rc;
    static thread_local EvalArgs a;
    memset(&a, 0, sizeof(a));
    int nl = 0, remap[256];
    for (int i = 0; i < 256; ++i) remap[i] = -1;
    int nc = 0;
    for (int L = 0; L < n_leaves; ++L) {
        if (L == mp_leaf) continue;
        const int ci = leaves[L].comp;
        if (remap[ci] < 0) {
            if (nc >= AGB_MAX_COMPONENTS)
                return set_err(AGB_ERR_UNSUPPORTED, "agb_adjoint_step: more than %d components",
                               AGB_MAX_COMPONENTS);
            if ((rc = comp_to_dev(comps[ci], a.comps[nc], AGB_PREC_FP64))) return rc;
            remap[ci] = nc++;
        }
        DevLeaf& d = a.leaves[nl++];
        d.comp = remap[ci];
        d.sigma = leaves[L].sigma;
        d.g0 = leaves[L].gamma[0]; d.g1 = leaves[L].gamma[1]; d.g2 = leaves[L].gamma[2];
        d.ampl = leaves[L].ampl;
        d.pad = 0;
    }
    a.n_leaves = nl;
    AdjStepPtrs q;
    q.x = x; q.vh = vh; q.lx = lx; q.lv = lv; q.gF = gF;
    q.dest = keep.dest; q.stage = keep.stage;
    q.n = n; q.stage_rec = drift ? 6 : 3; q.drift = drift ? 1 : 0; q.lv_cot = lv_cot ? 1 : 0;
    q.dt = dt; q.c = c; q.c_in = c_in; q.k = k; q.dt_drift = dt_drift;
    // 64-thread blocks, 8 per SM (the same 16 warps as 2 x 256): 1.3 % faster backward step
    adjoint_step_kernel<<<grid_for(n * 4), 64, 0, (cudaStream_t)stream>>>(a, q);
    return check_launch("adjoint_step_kernel");
}

extern "C" int agb_multipole_adjoint(const agb_component* comp, const agb_leaf* leaf,
                                     const double* xyz, int64_t n, int precision,
                                     const double* g_phi, const double* g_force, double* g_xyz,
                                     double* g_table, double* g_const, void* workspace,
                                     size_t workspace_bytes, void* stream)
{
    return multipole_adjoint_impl(comp, leaf, xyz, n, precision, g_phi, g_force, g_xyz, nullptr,
                                  g_table, g_const, workspace, workspace_bytes, stream);
}

extern "C" int agb_multipole_adjoint_force(const agb_component* comp, const agb_leaf* leaf,
                                           const double* xyz, int64_t n, int precision,
                                           const double* g_phi, const double* g_force,
                                           double* g_xyz, double* force, double* g_table,
                                           double* g_const, void* workspace,
                                           size_t workspace_bytes, void* stream)
{
    if (!force) return set_err(AGB_ERR_ARG, "agb_multipole_adjoint_force: force is null");
    return multipole_adjoint_impl(comp, leaf, xyz, n, precision, g_phi, g_force, g_xyz, force,
                                  g_table, g_const, workspace, workspace_bytes, stream);
}

// ---------------------------------------------------------------------------
// leapfrog adjoint: per-step vector updates
// ---------------------------------------------------------------------------
extern "C" int agb_adjoint_kick(double* lx, double* lv, const double* gx, double* gF, int64_t n,
                                double dt, double c, void* stream)
{
    if (n < 0) return set_err(AGB_ERR_ARG, "agb_adjoint_kick: negative count");
    if (n == 0) return AGB_OK;
    if (!lx || !lv || !gx || !gF) return set_err(AGB_ERR_ARG, "agb_adjoint_kick: null argument");
    const long long m = 3LL * n;
    adjoint_kick_kernel<<<grid_for(m), 256, 0, (cudaStream_t)stream>>>(lx, lv, gx, gF, m, dt, c);
    return check_launch("adjoint_kick_kernel");
}

extern "C" int agb_reverse_drift(double* x, double* vh, const double* F, int64_t n, double k,
                                 double dt, void* stream)
{
    if (n < 0) return set_err(AGB_ERR_ARG, "agb_reverse_drift: negative count");
    if (n == 0) return AGB_OK;
    if (!x || !vh || !F) return set_err(AGB_ERR_ARG, "agb_reverse_drift: null argument");
    const long long m = 3LL * n;
    reverse_drift_kernel<<<grid_for(m), 256, 0, (cudaStream_t)stream>>>(x, vh, F, m, k, dt);
    return check_launch("reverse_drift_kernel");
}

extern "C" int agb_cylspline_table_vjp(const agb_component* comp, const agb_leaf* leaf,
                                      const double* xyz, int64_t n, const double* g_phi,
                                      const double* g_force, double* g_cells, void* stream)
{
    if (!comp || !leaf || !g_cells)
        return set_err(AGB_ERR_ARG, "agb_cylspline_table_vjp: null argument");
    if (comp->kind != AGB_KIND_CYLSPLINE || comp->layout != 1)
        return set_err(AGB_ERR_ARG, "agb_cylspline_table_vjp: needs a cell-major CylSpline table");
    if (n < 0) return set_err(AGB_ERR_ARG, "agb_cylspline_table_vjp: negative point count");
    if (n == 0) return AGB_OK;
    if (!xyz) return set_err(AGB_ERR_ARG, "agb_cylspline_table_vjp: xyz is null");
    CSGradArgs g;
    memset(&g, 0, sizeof(g));
    int rc = comp_to_dev(*comp, g.c, AGB_PREC_FP64);
    if (rc) return rc;
    g.leaf.comp = 0; g.leaf.sigma = leaf->sigma; g.leaf.ampl = leaf->ampl;
    g.leaf.g0 = leaf->gamma[0]; g.leaf.g1 = leaf->gamma[1]; g.leaf.g2 = leaf->gamma[2];
    g.n = n; g.xyz = xyz; g.gphi = g_phi; g.gforce = g_force; g.grad = g_cells;
    cs_grad_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(g);
    return check_launch("cs_grad_kernel");
}

// ---------------------------------------------------------------------------
// agb_eval_static: the fused evaluation with its sorting scratch in a fixed
// device array of this library, for callers that must not allocate.
//
// Some host programs cannot let a library allocate device memory and cannot
// hand it scratch either: an N-body or orbit code that reserves the whole GPU
// for its own particle pool, a latency-critical loop that must never pay the
// device-wide synchronisation of cudaMalloc/cudaFree, or a plain C/Fortran
// caller whose interface only passes the arrays it already owns.  This entry
// point serves them.  The scratch lives in g_static_scratch below
// (AGB_STATIC_SCRATCH_BYTES = 32 MiB), which every GPU that loads this library
// holds until the process exits; it limits one call to AGB_STATIC_MAX_POINTS
// points.  Host code cannot use the array's name as a device address: the
// address is fetched with cudaGetSymbolAddress once per device (and once more
// after a device reset replaced its context), on the first call made with that
// device current, and that first call should be made before any stream capture
// begins.  All calls share the one array and it
// keeps whatever the last call left there (the bin counts that must start at
// zero are cleared by every call), so calls whose work overlaps on the GPU
// (other streams, other host threads) race on it: serialise them.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_static_scratch[AGB_STATIC_SCRATCH_BYTES];

// The largest call must fit: keys, permutation and sorted positions of
// AGB_STATIC_MAX_POINTS points plus the two bin arrays at their maximum
// (output staging is used only when it fits as well).
static_assert(2 * al256(4 * (size_t)AGB_STATIC_MAX_POINTS) + al256(24 * (size_t)AGB_STATIC_MAX_POINTS)
              + 2 * al256(4 * (size_t)AGB_MAX_BINS) <= (size_t)AGB_STATIC_SCRATCH_BYTES,
              "agb_eval_static: the fixed scratch array cannot hold a call of AGB_STATIC_MAX_POINTS");

// Id of the CUDA context current on this thread (0 when the driver cannot say).
// The driver entry points come through the runtime, so the library needs no
// link-time dependency on libcuda.
typedef CUresult (*agb_ctx_current_fn)(CUcontext*);
typedef CUresult (*agb_ctx_id_fn)(CUcontext, unsigned long long*);

static unsigned long long current_context_id()
{
    static std::once_flag once;
    static agb_ctx_current_fn get_current = nullptr;
    static agb_ctx_id_fn get_id = nullptr;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q)
                == cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_current = (agb_ctx_current_fn)f;
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q)
                == cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_id = (agb_ctx_id_fn)f;
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
        get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// The array's device address per device, with the context it was looked up in.
// A device reset (cudaDeviceReset) destroys the primary context and the module
// with it; the next call sees a new context id and looks the address up again.
struct StaticScratchSlot {
    std::mutex lock;
    unsigned long long ctx;
    void* addr;
};
static StaticScratchSlot g_static_slot[AGB_MAX_DEVICES];

static int static_scratch_address(int dev, void** out)
{
    StaticScratchSlot& s = g_static_slot[dev];
    std::lock_guard<std::mutex> guard(s.lock);
    const unsigned long long ctx = current_context_id();
    if (!s.addr || ctx == 0 || ctx != s.ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return set_err(AGB_ERR_DEVICE, "agb_eval_static: cudaGetSymbolAddress failed: %s",
                           cudaGetErrorString(e));
        s.addr = p;
        s.ctx = current_context_id();    // the lookup made the primary context current
    }
    *out = s.addr;
    return AGB_OK;
}

extern "C" int agb_eval_static(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                               int n_leaves, const double* xyz, int64_t n, int mode,
                               int precision, double* phi, double* grad, double* hess,
                               double* rho, int out_flags, void* stream)
{
    if (n > AGB_STATIC_MAX_POINTS)
        return set_err(AGB_ERR_UNSUPPORTED, "agb_eval_static: %lld points exceed its fixed scratch "
                       "limit of %d points (use agb_eval or agb_eval_ws)", (long long)n,
                       AGB_STATIC_MAX_POINTS);
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= AGB_MAX_DEVICES)
        return set_err(AGB_ERR_DEVICE, "agb_eval_static: no usable current CUDA device");
    void* scratch = nullptr;
    const int rc = static_scratch_address(dev, &scratch);
    if (rc) return rc;
    // eval_impl checks the scratch this call needs against the array's size
    return eval_impl(comps, n_comps, leaves, n_leaves, xyz, n, mode, precision, phi, grad, hess,
                     rho, out_flags, scratch, (size_t)AGB_STATIC_SCRATCH_BYTES, false, stream,
                     true);
}

// ---------------------------------------------------------------------------
// kernel-signature entries
// ---------------------------------------------------------------------------
static int mp_compat(int mode, const double* x, const double* y, const double* z,
                     const double* poly, double logr_min, double dlogr, double inv_dlogr,
                     int n_intervals, int n_lm, int lmax, const int* lm_l, const int* lm_m,
                     int log_scaling, double invPhi0, double inner_s, double inner_U,
                     double inner_W, double outer_s, double outer_U, double outer_W,
                     double* phi, double* grad, double* hess, double* rho, int N, void* stream)
{
    if (N < 0) return set_err(AGB_ERR_ARG, "negative N");
    if (N == 0) return AGB_OK;
    if (!x || !y || !z || !poly || !lm_l || !lm_m)
        return set_err(AGB_ERR_ARG, "multipole: null input pointer");
    if (n_lm < 1 || n_intervals < 1) return set_err(AGB_ERR_ARG, "multipole: empty tables");
    if (lmax > AGB_MAX_LMAX) return set_err(AGB_ERR_UNSUPPORTED, "lmax=%d exceeds %d", lmax, AGB_MAX_LMAX);
    if (!aligned16(poly)) return set_err(AGB_ERR_ARG, "poly must be 16-byte aligned");
    static thread_local EvalArgs a;
    memset(&a, 0, sizeof(a));
    a.n = N; a.soa = 1; a.x = x; a.y = y; a.z = z;
    a.phi = phi; a.grad = grad; a.hess = hess; a.rho = rho;
    DevComp& c = a.comps[0];
    c.kind = AGB_KIND_MULTIPOLE; c.n_lm = n_lm; c.n_int = n_intervals; c.lmax = lmax;
    c.log_scaling = log_scaling; c.layout = AGB_LAYOUT_HARMONIC_MAJOR; c.lm_split = 1;
    c.table = poly; c.lm = lm_l; c.lm_m = lm_m;
    const double p[10] = {logr_min, dlogr, inv_dlogr, invPhi0, inner_s, inner_U, inner_W,
                          outer_s, outer_U, outer_W};
    memcpy(c.p, p, sizeof(p));
    a.n_leaves = 1;
    a.leaves[0].comp = 0; a.leaves[0].sigma = 1.0; a.leaves[0].ampl = 1.0;
    return launch_mode(mode, AGB_PREC_FP64, a, (cudaStream_t)stream);
}

#define MP_SIG const double* x, const double* y, const double* z, const double* poly,       \
    double logr_min, double dlogr, double inv_dlogr, int n_intervals, int n_lm, int lmax,   \
    const int* lm_l, const int* lm_m, int log_scaling, double invPhi0, double inner_s,      \
    double inner_U, double inner_W, double outer_s, double outer_U, double outer_W
#define MP_FWD x, y, z, poly, logr_min, dlogr, inv_dlogr, n_intervals, n_lm, lmax, lm_l,    \
    lm_m, log_scaling, invPhi0, inner_s, inner_U, inner_W, outer_s, outer_U, outer_W

extern "C" int agb_multipole_potential(MP_SIG, double* phi_out, double* grad_out, int N, void* stream)
{
    (void)grad_out;
    if (!phi_out) return set_err(AGB_ERR_ARG, "phi_out is null");
    return mp_compat(AGB_MODE_POT, MP_FWD, phi_out, nullptr, nullptr, nullptr, N, stream);
}
extern "C" int agb_multipole_force(MP_SIG, double* phi_out, double* grad_out, int N, void* stream)
{
    if (!phi_out || !grad_out) return set_err(AGB_ERR_ARG, "phi_out/grad_out is null");
    return mp_compat(AGB_MODE_GRAD, MP_FWD, phi_out, grad_out, nullptr, nullptr, N, stream);
}
extern "C" int agb_multipole_hess(MP_SIG, double* phi_out, double* grad_out, double* hess_out,
                                  int N, void* stream)
{
    if (!phi_out || !grad_out || !hess_out) return set_err(AGB_ERR_ARG, "output pointer is null");
    return mp_compat(AGB_MODE_HESS, MP_FWD, phi_out, grad_out, hess_out, nullptr, N, stream);
}
extern "C" int agb_multipole_density(MP_SIG, double inv_4piG, double* rho_out, int N, void* stream)
{
    if (!rho_out) return set_err(AGB_ERR_ARG, "rho_out is null");
    if (inv_4piG != AGB_INV_4PIG && fabs(inv_4piG / AGB_INV_4PIG - 1.0) > 1e-12)
        return set_err(AGB_ERR_UNSUPPORTED, "inv_4piG must be 1/(4 pi G) in Agama units");
    return mp_compat(AGB_MODE_DENS, MP_FWD, nullptr, nullptr, nullptr, rho_out, N, stream);
}

static int cs_compat(int mode, const double* x, const double* y, const double* z, double Rscale,
                     const double* lR_grid, int nR, const double* lz_grid, int nz,
                     const double* node_arr, int n_harm, const int* m_arr, int mmax,
                     int log_scaling, const double* W_outer, double r0_outer, int lmax_outer,
                     int mmax_outer, double* phi, double* grad, double* hess, int N, void* stream)
{
    (void)mmax;
    if (N < 0) return set_err(AGB_ERR_ARG, "negative N");
    if (N == 0) return AGB_OK;
    if (!x || !y || !z || !lR_grid || !lz_grid || !node_arr || !m_arr || !W_outer)
        return set_err(AGB_ERR_ARG, "cylspline: null input pointer");
    if (nR < 2 || nz < 2 || n_harm < 1) return set_err(AGB_ERR_ARG, "cylspline: grid too small");
    if (lmax_outer > AGB_MAX_LMAX || mmax_outer > lmax_outer || mmax_outer < 0)
        return set_err(AGB_ERR_ARG, "cylspline: outer orders out of range");
    if (!aligned16(node_arr)) return set_err(AGB_ERR_ARG, "node_arr must be 16-byte aligned");
    static thread_local EvalArgs a;
    memset(&a, 0, sizeof(a));
    a.n = N; a.soa = 1; a.x = x; a.y = y; a.z = z;
    a.phi = phi; a.grad = grad; a.hess = hess;
    DevComp& c = a.comps[0];
    c.kind = AGB_KIND_CYLSPLINE; c.n_lm = n_harm; c.n_int = nR; c.nz = nz; c.lmax = lmax_outer;
    c.log_scaling = log_scaling; c.layout = 0; c.table = node_arr; c.lm = m_arr;
    c.grid_a = lR_grid; c.grid_b = lz_grid; c.extra = W_outer;
    c.p[0] = Rscale; c.p[1] = r0_outer; c.p[2] = (double)mmax_outer;
    a.n_leaves = 1;
    a.leaves[0].comp = 0; a.leaves[0].sigma = 1.0; a.leaves[0].ampl = 1.0;
    return launch_mode(mode, AGB_PREC_FP64, a, (cudaStream_t)stream);
}

#define CS_SIG const double* x, const double* y, const double* z, double Rscale,              \
    const double* lR_grid, int nR, const double* lz_grid, int nz, const double* node_arr,    \
    int n_harm, const int* m_arr, int mmax, int log_scaling, const double* W_outer,          \
    double r0_outer, int lmax_outer, int mmax_outer
#define CS_FWD x, y, z, Rscale, lR_grid, nR, lz_grid, nz, node_arr, n_harm, m_arr, mmax,     \
    log_scaling, W_outer, r0_outer, lmax_outer, mmax_outer

extern "C" int agb_cylspl_potential(CS_SIG, double* phi_out, int N, void* stream)
{
    if (!phi_out) return set_err(AGB_ERR_ARG, "phi_out is null");
    return cs_compat(AGB_MODE_POT, CS_FWD, phi_out, nullptr, nullptr, N, stream);
}
extern "C" int agb_cylspl_force(CS_SIG, double* phi_out, double* grad_out, int N, void* stream)
{
    if (!phi_out || !grad_out) return set_err(AGB_ERR_ARG, "output pointer is null");
    return cs_compat(AGB_MODE_GRAD, CS_FWD, phi_out, grad_out, nullptr, N, stream);
}
extern "C" int agb_cylspl_hess(CS_SIG, double* phi_out, double* grad_out, double* hess_out, int N,
                               void* stream)
{
    if (!phi_out || !grad_out || !hess_out) return set_err(AGB_ERR_ARG, "output pointer is null");
    return cs_compat(AGB_MODE_HESS, CS_FWD, phi_out, grad_out, hess_out, N, stream);
}

// ---------------------------------------------------------------------------
// batched work units (device work queue)
// ---------------------------------------------------------------------------
#include "batch.cuh"
