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
    const double* xyz;
    double* phi;
    double* grad;
    double* hess;
    double* rho;
};

template <int MODE, typename R>
__global__ void __launch_bounds__(256, (MODE == AGB_MODE_HESS) ? 1 : 2)
agb_batch_kernel(const __grid_constant__ BatchArgs a)
{
    __shared__ int s_tile;
    __shared__ int s_hist[AGB_BATCH_MAX_BINS], s_cur[AGB_BATCH_MAX_BINS];
    __shared__ unsigned short s_key[AGB_BATCH_SORT_MAX], s_order[AGB_BATCH_SORT_MAX];
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(a.counter, 1);
        __syncthreads();
        const int t = s_tile;
        __syncthreads();                  // every thread has read s_tile before it changes
        if (t >= a.n_tiles) return;
        const BatchTile T = a.tiles[t];
        const int l0 = a.unit_leaf[T.unit], l1 = a.unit_leaf[T.unit + 1];
        const BinKey K = a.ukey[T.unit];
        const int nb = K.n_int + 2;
        const bool sorted = K.n_int >= 0 && nb <= AGB_BATCH_MAX_BINS && T.count <= AGB_BATCH_SORT_MAX;
        if (sorted) {
            for (int q = threadIdx.x; q < nb; q += blockDim.x) s_hist[q] = 0;
            __syncthreads();
            for (int j = threadIdx.x; j < T.count; j += blockDim.x) {
                const long long i = T.start + j;
                const int k = bin_of(K, a.xyz[3 * i], a.xyz[3 * i + 1], a.xyz[3 * i + 2]);
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
            const long long i = T.start + (sorted ? (int)s_order[j] : j);
            const double x = a.xyz[3 * i], y = a.xyz[3 * i + 1], z = a.xyz[3 * i + 2];
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
            if (MODE == AGB_MODE_DENS) {
                a.rho[i] = rho;
                continue;
            }
            const double sg = (a.out_flags & AGB_OUT_NEGATE) ? -1.0 : 1.0;
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
        if (best >= 0) {
            const agb_component& c = comps[leaves[best].comp];
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
    const size_t bytes = o_k + 256;
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
    }
    free(hc); free(hl); free(ucost); free(hk); free(ht);
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

template <int MODE, typename R>
static int launch_batch(const BatchArgs& a, cudaStream_t st)
{
    static std::atomic<int> cache[AGB_MAX_DEVICES];   // resident blocks per SM, per device
    const int per_sm = blocks_per_sm(cache, agb_batch_kernel<MODE, R>, 256);
    const long long grid = std::min<long long>((long long)num_sms() * per_sm, a.n_tiles);
    agb_batch_kernel<MODE, R><<<(int)std::max<long long>(grid, 1), 256, 0, st>>>(a);
    return check_launch("agb_batch_kernel");
}

extern "C" int agb_batch_eval(const agb_batch* plan, const double* xyz, int mode, double* phi,
                              double* grad, double* hess, double* rho, int out_flags, void* stream)
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
    a.out_flags = out_flags; a.xyz = xyz;
    a.phi = phi; a.grad = grad; a.hess = hess; a.rho = rho;
    if (cudaMemsetAsync(plan->counter, 0, sizeof(int), st) != cudaSuccess)
        return set_err(AGB_ERR_DEVICE, "agb_batch_eval: reset of the work queue failed");
    const bool mixed = plan->precision == AGB_PREC_MIXED;
    switch (mode) {
    case AGB_MODE_POT:  return mixed ? launch_batch<AGB_MODE_POT, float>(a, st)  : launch_batch<AGB_MODE_POT, double>(a, st);
    case AGB_MODE_GRAD: return mixed ? launch_batch<AGB_MODE_GRAD, float>(a, st) : launch_batch<AGB_MODE_GRAD, double>(a, st);
    case AGB_MODE_HESS: return mixed ? launch_batch<AGB_MODE_HESS, float>(a, st) : launch_batch<AGB_MODE_HESS, double>(a, st);
    default:            return mixed ? launch_batch<AGB_MODE_DENS, float>(a, st) : launch_batch<AGB_MODE_DENS, double>(a, st);
    }
}
