// batch.cuh -- many independent (potential, point set) work units in one
// launch through a device work queue.  Included at the end of eval.cu (it uses
// that file's error helpers, descriptor conversion and component dispatch).
//
// A caller integrating hundreds of small systems (one potential per stream or
// satellite, a few thousand to a few hundred thousand particles each) would
// otherwise make one evaluation call per unit per step: hundreds of launches,
// most of them too small to fill 148 SMs.  Here the units are cut into tiles
// of at most tile_points points, sorted by estimated cost (points x per-point
// flops of the unit's leaves), and one persistent kernel -- as many blocks as
// fit on the GPU at once -- hands tiles out through an atomic counter: a block
// finishing a cheap tile immediately takes the next, so the expensive units
// (high lmax, many points) start first and the tail is made of small tiles.

// Within a tile the points are counting-sorted in shared memory by the radial
// interval of the unit's heaviest Multipole (the per-call binning of agb_eval,
// done here per tile with no global scratch), so a warp's lanes read the same
// interval's coefficients.
#define AGB_BATCH_SORT_MAX 8192        // largest tile that is sorted (34 KB of shared memory)
#define AGB_BATCH_MAX_BINS 256         // most intervals (+2) of a sorted unit

// Staging (AGB_OUT_STAGE, mixed precision, points pre-sorted): a tile of sorted
// points spans a run of intervals k0..k1 of its unit's keyed Multipole; one thread
// bulk-copies those rows of the FP32 table (contiguous in the interval-major layout,
// as many as fit in AGB_BATCH_STAGE_BYTES) into shared memory while the others wait
// on an mbarrier, and the walk of that component reads them there instead of
// through L1/L2.  A wait that gives up (bounded) records an error and the block reads
// global memory from then on.
#define AGB_BATCH_STAGE_BYTES (64 * 1024)
#define AGB_BATCH_STAGE_TRIES (1 << 22)
#include "bulk.cuh"

struct BatchTile {
    long long start;          // first point (row of xyz)
    int unit;
    int count;                // points in the tile
};

struct BatchArgs {
    const DevComp* comps;     // device [n_comps]
    const DevLeaf* leaves;    // device [n_leaves], comp indexes comps
    const int* unit_leaf;     // device [n_units + 1]
    const BatchTile* tiles;   // device [n_tiles], largest cost first
    const BinKey* ukey;       // device [n_units]: sort key of the unit (n_int < 0: none)
    int* counter;             // device, zero at launch
    int n_tiles;
    int out_flags;
    const double* xyz;        // presorted: the sorted copy of the points
    int xstride;              // doubles per point in xyz: 3 (the caller's), 4 (sorted copy)
    int presorted;            // xyz is the sorted copy made by this call's pre-sort
    double* phi;
    double* grad;
    double* hess;
    double* rho;
    const int* perm;          // presorted: sorted position -> row of the caller's arrays
    double* stage;            // presorted with room: per-position output records
    int* err;                 // ST: set to 1 when a staging wait gave up (sticky)
};

// ST: stage the keyed Multipole's interval rows of each tile (see above; FP32 only)
template <int MODE, typename R, bool ST = false>
__global__ void __launch_bounds__(256, (MODE == AGB_MODE_HESS) ? 1 : 2)
agb_batch_kernel(const __grid_constant__ BatchArgs a)
{
    __shared__ int s_tile;
    __shared__ int s_hist[AGB_BATCH_MAX_BINS], s_cur[AGB_BATCH_MAX_BINS];
    __shared__ unsigned short s_key[AGB_BATCH_SORT_MAX], s_order[AGB_BATCH_SORT_MAX];
    extern __shared__ __align__(128) float agb_batch_slab[];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_k0, s_k1, s_dead;
    unsigned phase = 0;
    if (ST) {
        if (threadIdx.x == 0) {
            mbar_init(&s_bar, 1);
            s_dead = 0;
        }
        __syncthreads();
    }
    for (;;) {
        if (ST) __syncthreads();          // the previous tile's reads of the slab are done
        if (threadIdx.x == 0) {
            s_tile = atomicAdd(a.counter, 1);
            if (ST) {
                // the tile's in-grid interval run from its first and last (sorted) point
                int k0 = 0, k1 = -1;
                const int tt = s_tile;
                if (tt < a.n_tiles && !s_dead) {
                    const BatchTile T = a.tiles[tt];
                    const BinKey K = a.ukey[T.unit];
                    const DevComp* kc = K.comp >= 0 ? &a.comps[K.comp] : nullptr;
                    if (kc && K.n_int > 0 && kc->kind == AGB_KIND_MULTIPOLE && kc->table32 &&
                        kc->structure != AGB_STRUCT_LIST && T.count > 0) {
                        const long long p0 = T.start, p1 = T.start + T.count - 1;
                        const int b0 = bin_of(K, a.xyz[a.xstride * p0], a.xyz[a.xstride * p0 + 1],
                                             a.xyz[a.xstride * p0 + 2]);
                        const int b1 = bin_of(K, a.xyz[a.xstride * p1], a.xyz[a.xstride * p1 + 1],
                                             a.xyz[a.xstride * p1 + 2]);
                        const long long row = 32LL * kc->n_lm;          // bytes per interval
                        if (b0 < K.n_int && row <= AGB_BATCH_STAGE_BYTES) {
                            k0 = b0;
                            k1 = b1 < K.n_int ? b1 : K.n_int - 1;
                            if (k1 < k0) k1 = k0;
                            const int fit = (int)(AGB_BATCH_STAGE_BYTES / row);
                            if (k1 - k0 + 1 > fit) k1 = k0 + fit - 1;
                            const unsigned bytes = (unsigned)((k1 - k0 + 1) * row);
                            // the previous tile's generic reads of the slab come first
                            fence_proxy_async_smem();
                            mbar_arrive_expect_tx(&s_bar, bytes);
                            bulk_copy_g2s(agb_batch_slab, kc->table32 + (long long)k0 * kc->n_lm * 8,
                                          bytes, &s_bar);
                        }
                    }
                }
                s_k0 = k0;
                s_k1 = k1;
            }
        }
        __syncthreads();
        const int t = s_tile;
        int k0 = 0, k1 = -1;
        if (ST) { k0 = s_k0; k1 = s_k1; }
        __syncthreads();                  // every thread has read s_tile before it changes
        if (t >= a.n_tiles) return;       // (no copy is issued for t >= n_tiles)
        if (ST && k1 >= k0) {
            // AGB_OUT_STAGE_GIVE_UP (tests of this path): give up at the first poll
            const bool ok = mbar_wait_bounded(&s_bar, phase,
                                              (a.out_flags & AGB_OUT_STAGE_GIVE_UP)
                                                  ? 0 : AGB_BATCH_STAGE_TRIES);
            phase ^= 1u;
            if (__syncthreads_or(!ok)) {  // gave up: read global memory from here on
                k1 = k0 - 1;
                if (threadIdx.x == 0) {
                    s_dead = 1;
                    if (a.err) atomicExch(a.err, 1);
                    // the copy in flight must land before the block can exit
                    mbar_wait_bounded(&s_bar, phase ^ 1u, AGB_BATCH_STAGE_TRIES);
                }
            }
        }
        const BatchTile T = a.tiles[t];
        const int l0 = a.unit_leaf[T.unit], l1 = a.unit_leaf[T.unit + 1];
        const BinKey K = a.ukey[T.unit];
        const int nb = K.n_int + 2;
        // points pre-sorted by agb_batch_eval_ws: a tile is a run of sorted positions
        // (AGB_OUT_NO_BINNING: the caller keeps the rows in interval order itself)
        const bool sorted = !a.presorted && !(a.out_flags & AGB_OUT_NO_BINNING) && K.n_int >= 0 &&
                            nb <= AGB_BATCH_MAX_BINS && T.count <= AGB_BATCH_SORT_MAX;
        if (sorted) {
            for (int q = threadIdx.x; q < nb; q += blockDim.x) s_hist[q] = 0;
            __syncthreads();
            for (int j = threadIdx.x; j < T.count; j += blockDim.x) {
                const long long i = T.start + j;
                const int k = bin_of(K, a.xyz[a.xstride * i], a.xyz[a.xstride * i + 1],
                                    a.xyz[a.xstride * i + 2]);
                s_key[j] = (unsigned short)k;
                atomicAdd(&s_hist[k], 1);
            }
            __syncthreads();
            if (threadIdx.x < 32) {        // exclusive scan of <= 256 bins by one warp
                const int lane = threadIdx.x, b0 = lane * (AGB_BATCH_MAX_BINS / 32);
                int loc = 0;
                for (int q = 0; q < AGB_BATCH_MAX_BINS / 32; ++q)
                    loc += (b0 + q < nb) ? s_hist[b0 + q] : 0;
                int inc = loc;
                for (int d = 1; d < 32; d <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, inc, d);
                    if (lane >= d) inc += v;
                }
                int run = inc - loc;
                for (int q = 0; q < AGB_BATCH_MAX_BINS / 32; ++q)
                    if (b0 + q < nb) {
                        s_cur[b0 + q] = run;
                        run += s_hist[b0 + q];
                    }
            }
            __syncthreads();
            for (int j = threadIdx.x; j < T.count; j += blockDim.x)
                s_order[atomicAdd(&s_cur[s_key[j]], 1)] = (unsigned short)j;
            __syncthreads();
        }
        for (int j = threadIdx.x; j < T.count; j += blockDim.x) {
            const long long pos = T.start + (sorted ? (int)s_order[j] : j);
            const long long i = a.perm ? (long long)__ldg(a.perm + pos) : pos;
            double x, y, z;
            if (a.xstride == 4) {           // the sorted copy: one aligned 32-byte record
                const double2 v = __ldg(reinterpret_cast<const double2*>(a.xyz + 4 * pos));
                x = v.x; y = v.y; z = __ldg(a.xyz + 4 * pos + 2);
            } else {
                x = a.xyz[3 * pos]; y = a.xyz[3 * pos + 1]; z = a.xyz[3 * pos + 2];
            }
            double phi = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, rho = 0.0;
            double h[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            for (int L = l0; L < l1; ++L) {
                const DevLeaf& lf = a.leaves[L];
                const DevComp& c = a.comps[lf.comp];
                PointOut o;
                o.phi = 0.0; o.rho = 0.0;
                o.g[0] = o.g[1] = o.g[2] = 0.0;
                #pragma unroll
                for (int q = 0; q < 6; ++q) o.h[q] = 0.0;
                if (ST && k1 >= k0 && lf.comp == K.comp)     // the staged component
                    multipole_point<MODE, R, true>(c, lf.sigma * x - lf.g0, lf.sigma * y - lf.g1,
                                                   lf.sigma * z - lf.g2, o, agb_batch_slab, k0, k1);
                else
                    eval_component<MODE, R, false>(c, lf.sigma * x - lf.g0, lf.sigma * y - lf.g1,
                                                   lf.sigma * z - lf.g2, o);
                const double A = lf.ampl;
                if (MODE == AGB_MODE_DENS) {
                    rho += (A * lf.sigma * lf.sigma) * o.rho;
                    continue;
                }
                phi += A * o.phi;
                if (MODE != AGB_MODE_POT) {
                    const double As = A * lf.sigma;
                    g0 += As * o.g[0]; g1 += As * o.g[1]; g2 += As * o.g[2];
                    if (MODE == AGB_MODE_HESS) {
                        const double As2 = As * lf.sigma;
                        #pragma unroll
                        for (int q = 0; q < 6; ++q) h[q] += As2 * o.h[q];
                    }
                }
            }
            const double sg = (a.out_flags & AGB_OUT_NEGATE) ? -1.0 : 1.0;
            if (a.stage) {               // sorted order: contiguous records, then a gather
                constexpr int REC = stage_rec(MODE);
                double* o = a.stage + REC * pos;
                if (MODE == AGB_MODE_DENS) { o[0] = rho; continue; }
                o[0] = phi;
                if (MODE != AGB_MODE_POT) { o[1] = sg * g0; o[2] = sg * g1; o[3] = sg * g2; }
                if (MODE == AGB_MODE_HESS) {
                    #pragma unroll
                    for (int q = 0; q < 6; ++q) o[4 + q] = sg * h[q];
                }
                continue;
            }
            if (MODE == AGB_MODE_DENS) {
                a.rho[i] = rho;
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
}

// Device-wide pre-sort of a batch (agb_batch_eval_ws): every unit's points by the
// radial interval of its sort key, each unit within its own rows (unit u owns
// global bins [ubin[u], ubin[u+1]) and the bins run unit by unit), so a tile --
// a run of sorted positions -- spans a few intervals instead of all of them and
// its blocks' table reads hit L1.  One block per tile; block-local histograms in
// shared memory, one global atomic per (tile, bin).
__global__ void __launch_bounds__(256)
batch_bin_count(const BatchTile* __restrict__ tiles, const BinKey* __restrict__ ukey,
                const int* __restrict__ ubin, const double* __restrict__ xyz,
                int* __restrict__ keys, int* __restrict__ counts)
{
    extern __shared__ int hist[];
    const BatchTile T = tiles[blockIdx.x];
    const BinKey K = ukey[T.unit];
    const int b0 = ubin[T.unit], nb = ubin[T.unit + 1] - b0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) hist[q] = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < T.count; j += blockDim.x) {
        const long long i = T.start + j;
        const int k = nb > 1 ? bin_of(K, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]) : 0;
        keys[i] = k;
        atomicAdd(&hist[k], 1);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nb; q += blockDim.x)
        if (hist[q]) atomicAdd(&counts[b0 + q], hist[q]);
}

// keys[i] becomes the sorted position of row i (the gather index of unpermute_kernel)
__global__ void __launch_bounds__(256)
batch_bin_scatter(const BatchTile* __restrict__ tiles, const int* __restrict__ ubin,
                  const double* __restrict__ xyz, int* __restrict__ keys,
                  int* __restrict__ cursor, int* __restrict__ perm, double* __restrict__ xs)
{
    extern __shared__ int sm[];
    const BatchTile T = tiles[blockIdx.x];
    const int b0 = ubin[T.unit], nb = ubin[T.unit + 1] - b0;
    int* hist = sm;
    int* base = sm + nb;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) hist[q] = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < T.count; j += blockDim.x) atomicAdd(&hist[keys[T.start + j]], 1);
    __syncthreads();
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
        const int c = hist[q];
        base[q] = c ? atomicAdd(&cursor[b0 + q], c) : 0;
        hist[q] = 0;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < T.count; j += blockDim.x) {
        const long long i = T.start + j;
        const int k = keys[i];
        const long long pos = (long long)base[k] + atomicAdd(&hist[k], 1);
        if (perm) perm[pos] = (int)i;
        keys[i] = (int)pos;
        if (xs) {          // 32-byte records: each write fills one whole sector
            double2* o = reinterpret_cast<double2*>(xs + 4 * pos);
            o[0] = make_double2(xyz[3 * i], xyz[3 * i + 1]);
            o[1] = make_double2(xyz[3 * i + 2], 0.0);
        }
    }
}

struct agb_batch {
    int device;
    int precision;
    int n_units;
    int n_tiles;
    int64_t n_points;
    void* mem;                // one device allocation: comps, leaves, unit_leaf, tiles, keys, counter
    const DevComp* comps;
    const DevLeaf* leaves;
    const int* unit_leaf;
    const BatchTile* tiles;
    const BinKey* ukey;
    int* counter;
    const int* ubin;          // device [n_units + 1]: first global bin of each unit
    int n_bins;               // bins of the pre-sort over all units (0: not pre-sortable)
    int max_unit_bins;        // largest unit's bin count (shared-memory histogram size)
};

// per-point flop estimate of a leaf (the roofline convention), for tile ordering
static double leaf_cost(const agb_component& c)
{
    if (c.kind == AGB_KIND_MULTIPOLE) return 48.0 * c.n_lm + 64.0;
    if (c.kind == AGB_KIND_CYLSPLINE) return 110.0 * c.n_lm + 80.0;
    return 30.0;
}

extern "C" int agb_batch_create(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                                const int32_t* unit_leaf_offsets, int n_units,
                                const int64_t* point_offsets, int precision, int tile_points,
                                agb_batch** out)
{
    if (!out) return set_err(AGB_ERR_ARG, "agb_batch_create: out is null");
    *out = nullptr;
    if (!comps || n_comps < 1 || !leaves || !unit_leaf_offsets || !point_offsets || n_units < 1)
        return set_err(AGB_ERR_ARG, "agb_batch_create: empty component, leaf or unit list");
    if (precision != AGB_PREC_FP64 && precision != AGB_PREC_MIXED)
        return set_err(AGB_ERR_ARG, "agb_batch_create: unknown precision %d", precision);
    if (tile_points == 0) tile_points = 4096;      // the largest sorted tile: fastest measured
    if (tile_points < 32 || tile_points > (1 << 20))
        return set_err(AGB_ERR_ARG, "agb_batch_create: tile_points %d outside [32, 2^20]", tile_points);
    if (unit_leaf_offsets[0] != 0 || point_offsets[0] != 0)
        return set_err(AGB_ERR_ARG, "agb_batch_create: offsets must start at 0");
    const int n_leaves = unit_leaf_offsets[n_units];
    for (int u = 0; u < n_units; ++u) {
        if (unit_leaf_offsets[u + 1] <= unit_leaf_offsets[u])
            return set_err(AGB_ERR_ARG, "agb_batch_create: unit %d has no leaves", u);
        if (unit_leaf_offsets[u + 1] - unit_leaf_offsets[u] > AGB_MAX_LEAVES)
            return set_err(AGB_ERR_UNSUPPORTED, "agb_batch_create: unit %d has more than %d leaves",
                           u, AGB_MAX_LEAVES);
        if (point_offsets[u + 1] < point_offsets[u])
            return set_err(AGB_ERR_ARG, "agb_batch_create: point offsets decrease at unit %d", u);
    }
    for (int L = 0; L < n_leaves; ++L)
        if (leaves[L].comp < 0 || leaves[L].comp >= n_comps)
            return set_err(AGB_ERR_ARG, "agb_batch_create: leaf %d refers to component %d of %d",
                           L, leaves[L].comp, n_comps);
    const int64_t n_points = point_offsets[n_units];

    // host images of the device arrays
    DevComp* hc = (DevComp*)calloc((size_t)n_comps, sizeof(DevComp));
    DevLeaf* hl = (DevLeaf*)calloc((size_t)n_leaves, sizeof(DevLeaf));
    double* ucost = (double*)calloc((size_t)n_units, sizeof(double));
    BinKey* hk = (BinKey*)calloc((size_t)n_units, sizeof(BinKey));
    if (!hc || !hl || !ucost || !hk) {
        free(hc); free(hl); free(ucost); free(hk);
        return set_err(AGB_ERR_DEVICE, "agb_batch_create: host allocation failed");
    }
    int rc = AGB_OK;
    for (int i = 0; i < n_comps && !rc; ++i) rc = comp_to_dev(comps[i], hc[i], precision);
    for (int L = 0; L < n_leaves && !rc; ++L) {
        hl[L].comp = leaves[L].comp;
        hl[L].sigma = leaves[L].sigma;
        hl[L].g0 = leaves[L].gamma[0]; hl[L].g1 = leaves[L].gamma[1]; hl[L].g2 = leaves[L].gamma[2];
        hl[L].ampl = leaves[L].ampl;
    }
    long long n_tiles = 0;
    for (int u = 0; u < n_units && !rc; ++u) {
        int best = -1;
        for (int L = unit_leaf_offsets[u]; L < unit_leaf_offsets[u + 1]; ++L) {
            const agb_component& c = comps[leaves[L].comp];
            ucost[u] += leaf_cost(c);
            if (c.kind == AGB_KIND_MULTIPOLE && c.n_lm >= 2 &&
                (best < 0 || c.n_lm > comps[leaves[best].comp].n_lm))
                best = L;
        }
        hk[u].n_int = -1;
        hk[u].comp = -1;
        if (best >= 0) {
            const agb_component& c = comps[leaves[best].comp];
            hk[u].comp = leaves[best].comp;
            hk[u].sigma = leaves[best].sigma;
            hk[u].g0 = leaves[best].gamma[0]; hk[u].g1 = leaves[best].gamma[1];
            hk[u].g2 = leaves[best].gamma[2];
            hk[u].logr_min = c.p[0];
            hk[u].inv_dlogr = c.p[2];
            hk[u].n_int = c.n_int;
        }
        n_tiles += (point_offsets[u + 1] - point_offsets[u] + tile_points - 1) / tile_points;
    }
    if (!rc && n_tiles > 0x7fffffffLL)
        rc = set_err(AGB_ERR_UNSUPPORTED, "agb_batch_create: %lld tiles exceed 2^31", n_tiles);
    BatchTile* ht = nullptr;
    if (!rc) {
        ht = (BatchTile*)malloc(sizeof(BatchTile) * (size_t)(n_tiles > 0 ? n_tiles : 1));
        if (!ht) rc = set_err(AGB_ERR_DEVICE, "agb_batch_create: host allocation failed");
    }
    if (!rc) {
        long long t = 0;
        for (int u = 0; u < n_units; ++u)
            for (int64_t s = point_offsets[u]; s < point_offsets[u + 1]; s += tile_points) {
                const int64_t e = std::min<int64_t>(point_offsets[u + 1], s + tile_points);
                ht[t].start = s; ht[t].unit = u; ht[t].count = (int)(e - s);
                ++t;
            }
        std::stable_sort(ht, ht + n_tiles, [&](const BatchTile& p, const BatchTile& q) {
            return p.count * ucost[p.unit] > q.count * ucost[q.unit];
        });
    }
    // one device allocation, 256-byte aligned sections
    const size_t o_c = 0;
    const size_t o_l = al256(o_c + sizeof(DevComp) * (size_t)n_comps);
    const size_t o_u = al256(o_l + sizeof(DevLeaf) * (size_t)n_leaves);
    const size_t o_t = al256(o_u + sizeof(int) * (size_t)(n_units + 1));
    const size_t o_y = al256(o_t + sizeof(BatchTile) * (size_t)(n_tiles > 0 ? n_tiles : 1));
    const size_t o_k = al256(o_y + sizeof(BinKey) * (size_t)n_units);
    const size_t o_b = o_k + 256;
    const size_t bytes = al256(o_b + sizeof(int) * (size_t)(n_units + 1));
    // global bins of the pre-sort: unit u owns n_int + 2 of them (1 without a key)
    int* hb = rc ? nullptr : (int*)malloc(sizeof(int) * (size_t)(n_units + 1));
    if (!rc && !hb) rc = set_err(AGB_ERR_DEVICE, "agb_batch_create: host allocation failed");
    long long n_bins = 0;
    int max_unit_bins = 1;
    for (int u = 0; u < n_units && !rc; ++u) {
        hb[u] = (int)std::min<long long>(n_bins, 0x7fffffffLL);
        const int nb = hk[u].n_int >= 0 ? hk[u].n_int + 2 : 1;
        n_bins += nb;
        max_unit_bins = std::max(max_unit_bins, nb);
    }
    if (!rc) hb[n_units] = (int)std::min<long long>(n_bins, 0x7fffffffLL);
    // (positions are 32-bit in the sort's keys and permutation)
    const bool presortable = n_bins < (1LL << 30) && max_unit_bins <= AGB_MAX_BINS &&
                             n_points < 0x7fffffffLL;
    agb_batch* p = nullptr;
    if (!rc) {
        p = (agb_batch*)calloc(1, sizeof(agb_batch));
        if (!p) rc = set_err(AGB_ERR_DEVICE, "agb_batch_create: host allocation failed");
    }
    if (!rc) {
        cudaGetDevice(&p->device);
        if (cudaMalloc(&p->mem, bytes) != cudaSuccess) {
            rc = set_err(AGB_ERR_DEVICE, "agb_batch_create: cannot allocate %zu device bytes", bytes);
            p->mem = nullptr;
        }
    }
    if (!rc) {
        char* m = (char*)p->mem;
        bool ok = cudaMemcpy(m + o_c, hc, sizeof(DevComp) * (size_t)n_comps, cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(m + o_l, hl, sizeof(DevLeaf) * (size_t)n_leaves, cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(m + o_u, unit_leaf_offsets, sizeof(int) * (size_t)(n_units + 1),
                              cudaMemcpyHostToDevice) == cudaSuccess;
        if (n_tiles > 0)
            ok = ok && cudaMemcpy(m + o_t, ht, sizeof(BatchTile) * (size_t)n_tiles,
                                  cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(m + o_y, hk, sizeof(BinKey) * (size_t)n_units,
                              cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemset(m + o_k, 0, 256) == cudaSuccess;
        ok = ok && cudaMemcpy(m + o_b, hb, sizeof(int) * (size_t)(n_units + 1),
                              cudaMemcpyHostToDevice) == cudaSuccess;
        if (!ok) rc = set_err(AGB_ERR_DEVICE, "agb_batch_create: upload of the plan failed");
        p->precision = precision;
        p->n_units = n_units;
        p->n_tiles = (int)n_tiles;
        p->n_points = n_points;
        p->comps = (const DevComp*)(m + o_c);
        p->leaves = (const DevLeaf*)(m + o_l);
        p->unit_leaf = (const int*)(m + o_u);
        p->tiles = (const BatchTile*)(m + o_t);
        p->ukey = (const BinKey*)(m + o_y);
        p->counter = (int*)(m + o_k);
        p->ubin = (const int*)(m + o_b);
        p->n_bins = presortable ? (int)n_bins : 0;
        p->max_unit_bins = max_unit_bins;
    }
    free(hc); free(hl); free(ucost); free(hk); free(ht); free(hb);
    if (rc) {
        if (p) {
            if (p->mem) cudaFree(p->mem);
            free(p);
        }
        return rc;
    }
    *out = p;
    return AGB_OK;
}

extern "C" int64_t agb_batch_points(const agb_batch* plan) { return plan ? plan->n_points : -1; }
extern "C" int agb_batch_tiles(const agb_batch* plan) { return plan ? plan->n_tiles : -1; }

extern "C" void agb_batch_destroy(agb_batch* plan)
{
    if (!plan) return;
    if (plan->mem) {
        int cur = 0;
        cudaGetDevice(&cur);
        if (cur != plan->device) cudaSetDevice(plan->device);
        cudaFree(plan->mem);
        if (cur != plan->device) cudaSetDevice(cur);
    }
    free(plan);
}

// Scratch of the pre-sort: keys and perm (4 B per point each), the sorted copy of
// the points (32-byte records: x, y, z, pad), the bin counters and cursors, then
// (optional) the sorted-order output records.
static size_t batch_ws_bytes(const agb_batch* p)
{
    const size_t n = (size_t)p->n_points;
    return 2 * al256(4 * n) + al256(32 * n) + 2 * al256(4 * (size_t)p->n_bins);
}

extern "C" size_t agb_batch_workspace_bytes(const agb_batch* plan, int mode)
{
    if (!plan || plan->n_bins == 0 || plan->n_tiles == 0) return 0;
    if (mode != AGB_MODE_POT && mode != AGB_MODE_GRAD && mode != AGB_MODE_HESS &&
        mode != AGB_MODE_DENS)
        return 0;
    return batch_ws_bytes(plan) + al256(8 * (size_t)stage_rec(mode) * (size_t)plan->n_points);
}

template <int MODE, typename R>
static int launch_batch(const BatchArgs& a, cudaStream_t st)
{
    // staging: FP32 tables, points pre-sorted by this call.  (Rows an integrator keeps
    // in the order of its run's start drift apart along r: a tile's first and last
    // points then bound its intervals less well, and 100 config-4 leapfrog steps took
    // 1363 ms staged against 1307 ms unstaged.)
    const bool stage = std::is_same<R, float>::value && (a.out_flags & AGB_OUT_STAGE) && a.presorted;
    if (stage) {
        static std::atomic<int> cache_st[AGB_MAX_DEVICES];
        const int dev = current_device();
        int per_sm = cache_st[dev].load(std::memory_order_relaxed);
        if (per_sm == 0) {
            cudaFuncSetAttribute(agb_batch_kernel<MODE, R, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, AGB_BATCH_STAGE_BYTES);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, agb_batch_kernel<MODE, R, true>,
                                                              256, AGB_BATCH_STAGE_BYTES) != cudaSuccess ||
                per_sm < 1)
                per_sm = 1;
            cache_st[dev].store(per_sm, std::memory_order_relaxed);
        }
        const long long grid = std::min<long long>((long long)num_sms() * per_sm, a.n_tiles);
        agb_batch_kernel<MODE, R, true><<<(int)std::max<long long>(grid, 1), 256,
                                          AGB_BATCH_STAGE_BYTES, st>>>(a);
        return check_launch("agb_batch_kernel");
    }
    static std::atomic<int> cache[AGB_MAX_DEVICES];   // resident blocks per SM, per device
    const int per_sm = blocks_per_sm(cache, agb_batch_kernel<MODE, R>, 256);
    const long long grid = std::min<long long>((long long)num_sms() * per_sm, a.n_tiles);
    agb_batch_kernel<MODE, R><<<(int)std::max<long long>(grid, 1), 256, 0, st>>>(a);
    return check_launch("agb_batch_kernel");
}

// 1 when a staged batch kernel of this plan gave up waiting for a bulk copy (its
// blocks then read global memory; results are unaffected), else 0; -1 on error
extern "C" int agb_batch_stage_errors(const agb_batch* plan)
{
    if (!plan) return set_err(AGB_ERR_ARG, "agb_batch_stage_errors: plan is null");
    int v = 0;
    if (cudaMemcpy(&v, plan->counter + 1, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_err(AGB_ERR_DEVICE, "agb_batch_stage_errors: read failed");
    return v;
}

static std::atomic<unsigned long long> g_batch_bin_attr{0};     // one bit per device

// the counting sort of the pre-sort: perm (sorted position -> row), keys (row -> sorted
// position), xs (the sorted copy of the points, when given)
static int batch_sort(const agb_batch* p, const double* xyz, int* keys, int* perm, double* xs,
                      int* counts, cudaStream_t st)
{
    int* cursor = counts + p->n_bins;
    const unsigned long long bit = 1ull << current_device();
    if (!(g_batch_bin_attr.load(std::memory_order_acquire) & bit)) {
        cudaFuncSetAttribute(batch_bin_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             4 * AGB_MAX_BINS);
        cudaFuncSetAttribute(batch_bin_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             8 * AGB_MAX_BINS);
        g_batch_bin_attr.fetch_or(bit, std::memory_order_release);
    }
    if (cudaMemsetAsync(counts, 0, 4 * (size_t)p->n_bins, st) != cudaSuccess)
        return set_err(AGB_ERR_DEVICE, "agb_batch_eval_ws: memset of the bin counts failed");
    const size_t h = 4 * (size_t)p->max_unit_bins;
    batch_bin_count<<<p->n_tiles, 256, h, st>>>(p->tiles, p->ukey, p->ubin, xyz, keys, counts);
    int rc = check_launch("batch_bin_count");
    if (rc) return rc;
    bin_scan<<<1, 1024, 0, st>>>(counts, cursor, p->n_bins);
    if ((rc = check_launch("bin_scan"))) return rc;
    batch_bin_scatter<<<p->n_tiles, 256, 2 * h, st>>>(p->tiles, p->ubin, xyz, keys, cursor, perm, xs);
    return check_launch("batch_bin_scatter");
}

// with_perm false: the outputs go through sorted-order records and keys (row ->
// sorted position), so the permutation is not written
static int batch_presort(const agb_batch* p, const double* xyz, char* ws, BatchArgs& a,
                         bool with_perm, cudaStream_t st)
{
    const size_t n = (size_t)p->n_points;
    int* keys = (int*)ws;
    int* perm = with_perm ? (int*)(ws + al256(4 * n)) : nullptr;
    double* xs = (double*)(ws + 2 * al256(4 * n));
    int* counts = (int*)(ws + 2 * al256(4 * n) + al256(32 * n));
    const int rc = batch_sort(p, xyz, keys, perm, xs, counts, st);
    if (rc) return rc;
    a.xyz = xs;
    a.xstride = 4;
    a.perm = perm;
    a.presorted = 1;
    return AGB_OK;
}

extern "C" size_t agb_batch_sort_workspace_bytes(const agb_batch* plan)
{
    if (!plan || plan->n_bins == 0 || plan->n_tiles == 0) return 0;
    return al256(4 * (size_t)plan->n_points) + al256(8 * (size_t)plan->n_bins);
}

extern "C" int agb_batch_sort(const agb_batch* plan, const double* xyz, int32_t* perm,
                              void* workspace, size_t workspace_bytes, void* stream)
{
    if (!plan) return set_err(AGB_ERR_ARG, "agb_batch_sort: plan is null");
    if (plan->n_tiles == 0) return AGB_OK;
    if (plan->n_bins == 0)
        return set_err(AGB_ERR_UNSUPPORTED, "agb_batch_sort: the plan's units cannot be sorted "
                       "(more than %d intervals or 2^31 points)", AGB_MAX_BINS - 2);
    if (!xyz || !perm) return set_err(AGB_ERR_ARG, "agb_batch_sort: null array");
    const size_t need = agb_batch_sort_workspace_bytes(plan);
    if (!workspace || ((uintptr_t)workspace & 255u) || workspace_bytes < need)
        return set_err(AGB_ERR_ARG, "agb_batch_sort: a 256-byte aligned workspace of %zu bytes "
                       "is required", need);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != plan->device)
        return set_err(AGB_ERR_ARG, "agb_batch_sort: plan lives on device %d, current is %d",
                       plan->device, cur);
    char* ws = (char*)workspace;
    return batch_sort(plan, xyz, (int*)ws, (int*)perm, nullptr,
                      (int*)(ws + al256(4 * (size_t)plan->n_points)), (cudaStream_t)stream);
}

extern "C" int agb_batch_eval(const agb_batch* plan, const double* xyz, int mode, double* phi,
                              double* grad, double* hess, double* rho, int out_flags, void* stream)
{
    return agb_batch_eval_ws(plan, xyz, mode, phi, grad, hess, rho, out_flags, nullptr, 0, stream);
}

extern "C" int agb_batch_eval_ws(const agb_batch* plan, const double* xyz, int mode, double* phi,
                                 double* grad, double* hess, double* rho, int out_flags,
                                 void* workspace, size_t workspace_bytes, void* stream)
{
    if (!plan) return set_err(AGB_ERR_ARG, "agb_batch_eval: plan is null");
    switch (mode) {
    case AGB_MODE_POT:  if (!phi) return set_err(AGB_ERR_ARG, "agb_batch_eval: phi is null"); break;
    case AGB_MODE_GRAD: if (!grad) return set_err(AGB_ERR_ARG, "agb_batch_eval: grad is null"); break;
    case AGB_MODE_HESS: if (!hess) return set_err(AGB_ERR_ARG, "agb_batch_eval: hess is null"); break;
    case AGB_MODE_DENS: if (!rho) return set_err(AGB_ERR_ARG, "agb_batch_eval: rho is null"); break;
    default: return set_err(AGB_ERR_ARG, "agb_batch_eval: mode %d is not batched", mode);
    }
    if (plan->n_tiles == 0) return AGB_OK;
    if (!xyz) return set_err(AGB_ERR_ARG, "agb_batch_eval: xyz is null");
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != plan->device)
        return set_err(AGB_ERR_ARG, "agb_batch_eval: plan lives on device %d, current is %d",
                       plan->device, cur);
    cudaStream_t st = (cudaStream_t)stream;
    BatchArgs a;
    a.comps = plan->comps; a.leaves = plan->leaves; a.unit_leaf = plan->unit_leaf;
    a.tiles = plan->tiles; a.ukey = plan->ukey; a.counter = plan->counter;
    a.n_tiles = plan->n_tiles;
    a.out_flags = out_flags; a.xyz = xyz; a.xstride = 3; a.presorted = 0;
    a.phi = phi; a.grad = grad; a.hess = hess; a.rho = rho;
    a.perm = nullptr; a.stage = nullptr;
    a.err = plan->counter + 1;            // the word after the queue counter (sticky)
    int rc = AGB_OK;
    const int* dest = nullptr;
    if (workspace && plan->n_bins > 0 && !(out_flags & AGB_OUT_NO_BINNING)) {
        const size_t need = batch_ws_bytes(plan);
        if (((uintptr_t)workspace & 255u) || workspace_bytes < need)
            return set_err(AGB_ERR_ARG, "agb_batch_eval_ws: workspace of %zu bytes (256-byte "
                           "aligned) is smaller than the %zu bytes of the pre-sort",
                           workspace_bytes, need);
        const bool room = workspace_bytes >= agb_batch_workspace_bytes(plan, mode);
        if ((rc = batch_presort(plan, xyz, (char*)workspace, a, !room, st))) return rc;
        if (room) {
            a.stage = (double*)((char*)workspace + need);
            dest = (const int*)workspace;
        }
    }
    if (cudaMemsetAsync(plan->counter, 0, sizeof(int), st) != cudaSuccess)
        return set_err(AGB_ERR_DEVICE, "agb_batch_eval: reset of the work queue failed");
    const bool mixed = plan->precision == AGB_PREC_MIXED;
    switch (mode) {
    case AGB_MODE_POT:  rc = mixed ? launch_batch<AGB_MODE_POT, float>(a, st)  : launch_batch<AGB_MODE_POT, double>(a, st); break;
    case AGB_MODE_GRAD: rc = mixed ? launch_batch<AGB_MODE_GRAD, float>(a, st) : launch_batch<AGB_MODE_GRAD, double>(a, st); break;
    case AGB_MODE_HESS: rc = mixed ? launch_batch<AGB_MODE_HESS, float>(a, st) : launch_batch<AGB_MODE_HESS, double>(a, st); break;
    default:            rc = mixed ? launch_batch<AGB_MODE_DENS, float>(a, st) : launch_batch<AGB_MODE_DENS, double>(a, st); break;
    }
    if (rc || !a.stage) return rc;
    const long long n = plan->n_points;
    switch (mode) {
    case AGB_MODE_POT:  unpermute_kernel<AGB_MODE_POT><<<grid_for(n), 256, 0, st>>>(dest, a.stage, n, phi, grad, hess, rho); break;
    case AGB_MODE_GRAD: unpermute_kernel<AGB_MODE_GRAD><<<grid_for(n), 256, 0, st>>>(dest, a.stage, n, phi, grad, hess, rho); break;
    case AGB_MODE_HESS: unpermute_kernel<AGB_MODE_HESS><<<grid_for(n), 256, 0, st>>>(dest, a.stage, n, phi, grad, hess, rho); break;
    default:            unpermute_kernel<AGB_MODE_DENS><<<grid_for(n), 256, 0, st>>>(dest, a.stage, n, phi, grad, hess, rho); break;
    }
    return check_launch("unpermute_kernel");
}
