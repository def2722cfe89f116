// mgp_batch.cuh -- many independent problems solved together (included by mgp_engine.cu).
//
// A batch holds refinement solvers (FP64 level 0 + FP32/FP64 correction hierarchy), one
// per problem, of any sizes and level counts.  One refinement step for every active problem
// is a fixed sequence of launches; each launch is ONE persistent kernel over a work list of
// (problem, tile) items, so a level operation runs once for all problems that take part in
// it, whatever their shapes.
//
// Alignment by depth.  Level l of a problem with top depth T = levels-1 sits at depth
// d = T - l (the coarsest level is depth 0).  The reference's F-cycle (include/fcycle.h:13-97)
// on a problem of top T is
//     FF(T) = relax(T), setup(T), FF(T-1), P(T), V(T),        FF(0) = V(0) = relax(0),
// so the F-cycle of a top-(T-1) problem is exactly the stretch of a top-T problem's cycle
// between setup(T) and P(T).  The batched cycle therefore runs FF(Dmax) once, and at every
// operation at depth d takes part every problem whose own FF(d) is running there: the
// problems with top >= d inside BFF(d), and only those of the enclosing set inside a V-cycle.
// Each problem sees exactly its own F-cycle (the same operations in the same order).

// Blocks per SM that one batched launch's work list is cut into (shared among its problems by
// points); a compile-time knob.
#ifndef MGP_BATCH_BLOCKS_PER_SM
#define MGP_BATCH_BLOCKS_PER_SM 8
#endif

// ---- generic persistent work-list kernel -------------------------------------------------
template <typename Args>
struct BatchItem {
    Args a;
    int tile_start;  // first global tile of this item
    int gx, gy;      // tile grid of this item
    int pad;
};

template <typename Args, typename Tile>
__global__ void __launch_bounds__(256) kb_run(const BatchItem<Args>* __restrict__ items, int n, int total) {
    pdl_begin();
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
        int lo = 0, hi = n - 1;  // last item whose tile_start <= tile
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].tile_start <= tile) lo = mid;
            else hi = mid - 1;
        }
        const BatchItem<Args>& it = items[lo];
        const int local = tile - it.tile_start;
        Tile::run(it.a, local % it.gx, local / it.gx, it.gx);
        __syncthreads();  // shared reduction scratch is reused by the next tile
    }
}

template <typename T, int OP>
struct TStencil {
    using Args = StencilArgs<T>;
    static __device__ __forceinline__ void run(const Args& a, int bx, int by, int) { stencil_tile<T, OP, false>(a, bx, by); }
};
template <typename T>
struct TRestrict {
    using Args = RestrictArgs<T>;
    static __device__ __forceinline__ void run(const Args& a, int bx, int by, int) { restrict_tile(a, bx, by); }
};
template <typename T>
struct TBc {
    using Args = BcRestrictArgs<T>;
    static __device__ __forceinline__ void run(const Args& a, int bx, int by, int gx) { bc_restrict_tile(a, bx, by, gx); }
};
template <typename T>
struct TProlongAdd {
    using Args = ProlongArgs<T>;
    static __device__ __forceinline__ void run(const Args& a, int bx, int by, int) { prolong_tile<T, true>(a, bx, by); }
};
template <typename Ti>
struct TUpdate {
    using Args = UpdateArgs<double, Ti>;
    static __device__ __forceinline__ void run(const Args& a, int bx, int by, int) { refine_update_tile(a, bx, by); }
};
template <typename Ti>
struct TRefRes {
    using Args = RefineArgs<double, Ti>;
    static __device__ __forceinline__ void run(const Args& a, int bx, int by, int) {
        refine_residual_tile<double, Ti, false>(a, bx, by);
    }
};

namespace {

// ---- host-side launch list ----------------------------------------------------------------
struct BatchLaunch {
    size_t offset = 0;  // byte offset of this launch's items in the item buffer
    int n = 0, total = 0, grid = 0;
    void (*fn)(const void* items, int n, int total, int grid, cudaStream_t st) = nullptr;
};

template <typename Tile>
void launch_items(const void* items, int n, int total, int grid, cudaStream_t st) {
    launch_pdl(kb_run<typename Tile::Args, Tile>, dim3(grid), dim3(kThreads), 0, st,
               (const BatchItem<typename Tile::Args>*)items, n, total);
}

struct ScheduleBuilder {
    std::vector<unsigned char> bytes;
    std::vector<BatchLaunch> launches;
    int sms = 148;
    template <typename Tile>
    void add(const std::vector<BatchItem<typename Tile::Args>>& items) {
        if (items.empty()) return;
        using Item = BatchItem<typename Tile::Args>;
        BatchLaunch L;
        L.offset = (bytes.size() + 255) / 256 * 256;
        bytes.resize(L.offset + items.size() * sizeof(Item));
        memcpy(bytes.data() + L.offset, items.data(), items.size() * sizeof(Item));
        L.n = (int)items.size();
        L.total = 0;
        for (auto& it : items) L.total = std::max(L.total, it.tile_start + it.gx * it.gy);
        L.grid = std::max(1, std::min(L.total, sms * 8));
        L.fn = &launch_items<Tile>;
        launches.push_back(L);
    }
};

template <typename Args>
void push_item(std::vector<BatchItem<Args>>& v, const Args& a, int gx, int gy) {
    BatchItem<Args> it;
    it.a = a;
    it.tile_start = v.empty() ? 0 : v.back().tile_start + v.back().gx * v.back().gy;
    it.gx = gx;
    it.gy = gy;
    it.pad = 0;
    v.push_back(it);
}

// Kernel arguments and tile grid of one stencil sweep, as launch_stencil computes them.
template <typename T, int OP>
StencilArgs<T> stencil_args(mgp_solver* s, int l, const void* src, void* dst, T omega, int colour, int* gx, int* gy,
                            int target) {
    LevelState& L = s->lv[l];
    StencilArgs<T> a;
    a.G = L.G;
    a.src = (const T*)src;
    a.dst = (T*)dst;
    a.f = (const T*)L.f;
    a.F = faces_of<T>(s, l);
    a.two_h = (T)(2.0 * L.h);
    a.hsq = (T)(L.h * L.h);
    a.one_omega = (T)(1.0 - omega);
    a.omega_sixth = (T)(omega / 6.0);
    hsq_terms(a.hsq, a.inv_hsq, a.hsq_pow2);
    a.colour = colour;
    a.norm = nullptr;
    constexpr int V = VecT<T>::V;
    const int plane = L.G.ny * ((L.G.nz + V - 1) / V);
    const int bx = (plane + kThreads - 1) / kThreads;
    int chunks = 1;
    if (OP != OP_GS_COLUMN) {
        // no short marches here: on the 256-problem batch they cost 13% (FP64 275 -> 240, FP32
        // 447 -> 383 solves/s); the persistent work list does better with fewer, longer tiles
        chunks = std::max(1, std::min((target + bx - 1) / bx, L.G.nx));
    }
    a.ichunk = (L.G.nx + chunks - 1) / chunks;
    chunks = (L.G.nx + a.ichunk - 1) / a.ichunk;
    *gx = bx;
    *gy = chunks;
    return a;
}

}  // namespace

// ---- the batch ----------------------------------------------------------------------------
struct BatchProblem {
    int id = -1;
    mgp_solver* s = nullptr;  // refinement solver
    int top = 0;              // levels - 1
    double fnorm = 0.0, rel = 0.0, first_rel = 0.0;
    int64_t iters = 0;
    bool started = false, active = true;
    int slot = 0;             // norm slot
};

struct mgp_batch {
    mgp_batch_desc desc{};
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<BatchProblem> probs;
    int next_id = 0;
    unsigned long long* d_norms = nullptr;  // one slot per problem
    unsigned long long* h_norms = nullptr;
    int slots = 0;
    // cached schedule of one refinement step for the current active set
    bool dirty = true;
    std::vector<uint64_t> sched_state;  // inner state bits the schedule was built from
    std::vector<uint64_t> post_state;
    void* d_items = nullptr;
    size_t d_items_bytes = 0;
    std::vector<BatchLaunch> launches;
    cudaGraphExec_t graph = nullptr;
    int64_t launches_total = 0;
    int64_t launches_last = 0;  // launches of the latest non-empty schedule
    int stable_steps = 0;       // steps run since the active set last changed
    // Problems allocate their hierarchies from this pool in the batch stream's order: memory
    // of a retired problem goes back to the pool, not to the driver, so admitting and
    // retiring never synchronise the device.  h_slab: 64 pinned bytes per slot.
    cudaMemPool_t pool = nullptr;
    unsigned long long* h_slab = nullptr;
};

namespace {

void batch_free_schedule(mgp_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->launches.clear();
}

// Items of one refinement step for the active problems (see the file comment).
template <typename Ti>
int build_step(mgp_batch* b, ScheduleBuilder& sb) {
    std::vector<BatchProblem*> act;
    for (auto& p : b->probs)
        if (p.active && p.started) act.push_back(&p);
    if (act.empty()) return MGP_OK;
    int dmax = 0;
    for (auto* p : act) dmax = std::max(dmax, p->top);
    const double omega = b->desc.omega < 0 ? (b->desc.relaxation == MGP_JACOBI ? 6.0 / 7.0 : 8.0 / 9.0) : b->desc.omega;
    const int64_t ns = b->desc.nsmooth;
    const bool jac = b->desc.relaxation == MGP_JACOBI;
    // Blocks of a problem's march in one batched launch: its share, by points, of SMs*8 blocks
    // for the whole launch.  Few problems get many short marches each; many problems get few
    // long ones, as the batch supplies the parallelism (256-problem batch on B200: 0.99 s / 0.64 s
    // per FP64 / FP32 solve against 1.06 s / 0.69 s with a fixed SMs*2 blocks per problem).
    const double launch_blocks = (double)sm_count(b->device) * MGP_BATCH_BLOCKS_PER_SM;
    auto shares = [&](const std::vector<BatchProblem*>& set, int d) {
        std::vector<int> t(set.size());
        double tot = 0.0;
        for (auto* p : set) {
            const Geom& G = p->s->inner->lv[p->top - d].G;
            tot += (double)G.nx * G.ny * G.nz;
        }
        for (size_t i = 0; i < set.size(); i++) {
            const Geom& G = set[i]->s->inner->lv[set[i]->top - d].G;
            t[i] = std::max(1, (int)(launch_blocks * ((double)G.nx * G.ny * G.nz) / tot + 0.5));
        }
        return t;
    };
    auto members = [&](int thr) {
        std::vector<BatchProblem*> m;
        for (auto* p : act)
            if (p->top >= thr) m.push_back(p);
        return m;
    };
    // level operations, each one batched launch over `set` at depth d
    auto relax = [&](int d, const std::vector<BatchProblem*>& set) {
        const int sweeps = jac ? (int)ns : (int)(2 * ns);
        const std::vector<int> tgt = shares(set, d);
        for (int sw = 0; sw < sweeps; sw++) {
            std::vector<BatchItem<StencilArgs<Ti>>> items, items_col;
            for (size_t pi = 0; pi < set.size(); pi++) {
                BatchProblem* p = set[pi];
                mgp_solver* in = p->s->inner;
                const int l = p->top - d;
                int gx, gy;
                if (jac) {
                    in->lv[l].cur ^= 1;
                    auto a = stencil_args<Ti, OP_JACOBI>(in, l, uprev_ptr(in, l), u_ptr(in, l), (Ti)omega, 0, &gx, &gy,
                                                         tgt[pi]);
                    push_item(items, a, gx, gy);
                } else {
                    const int colour = in->gs_alternate ? 0 : 1;
                    if (in->lv[l].gs_column) {
                        auto a = stencil_args<Ti, OP_GS_COLUMN>(in, l, u_ptr(in, l), u_ptr(in, l), (Ti)omega, colour,
                                                                &gx, &gy, tgt[pi]);
                        push_item(items_col, a, gx, gy);
                    } else {
                        auto a = stencil_args<Ti, OP_GS>(in, l, u_ptr(in, l), u_ptr(in, l), (Ti)omega, colour, &gx, &gy,
                                                         tgt[pi]);
                        push_item(items, a, gx, gy);
                    }
                    in->gs_alternate = !in->gs_alternate;
                }
            }
            if (jac) sb.add<TStencil<Ti, OP_JACOBI>>(items);
            else {
                sb.add<TStencil<Ti, OP_GS>>(items);
                sb.add<TStencil<Ti, OP_GS_COLUMN>>(items_col);
            }
        }
    };
    auto setup = [&](int d, const std::vector<BatchProblem*>& set) {
        std::vector<BatchItem<StencilArgs<Ti>>> res;
        std::vector<BatchItem<RestrictArgs<Ti>>> rst;
        std::vector<BatchItem<BcRestrictArgs<Ti>>> bcs;
        const std::vector<int> tgt = shares(set, d);
        for (size_t pi = 0; pi < set.size(); pi++) {
            BatchProblem* p = set[pi];
            mgp_solver* in = p->s->inner;
            const int l = p->top - d;
            int gx, gy;
            auto a = stencil_args<Ti, OP_RESIDUAL>(in, l, u_ptr(in, l), in->lv[l].r, Ti(0), 0, &gx, &gy, tgt[pi]);
            push_item(res, a, gx, gy);
            long long n = 0;
            auto ra = restrict_args<Ti>(in, l, true, &n);
            const Geom& Gc = in->lv[l + 1].G;
            push_item(rst, ra, (Gc.ny * Gc.nz + kThreads - 1) / kThreads, Gc.nx);
            bool any = false;
            auto ba = bc_args<Ti>(in, l, &any);
            if (any) {
                long long nmax = 1;
                for (int f = 0; f < 6; f++) {
                    const int64_t* fs = in->lv[l + 1].face_shape[f];
                    nmax = std::max(nmax, (long long)(fs[0] * fs[1] * fs[2]));
                }
                push_item(bcs, ba, (int)((nmax + kThreads - 1) / kThreads), 6);
            }
        }
        sb.add<TStencil<Ti, OP_RESIDUAL>>(res);
        sb.add<TRestrict<Ti>>(rst);
        sb.add<TBc<Ti>>(bcs);
    };
    auto prolong = [&](int d, const std::vector<BatchProblem*>& set) {
        std::vector<BatchItem<ProlongArgs<Ti>>> items;
        constexpr int V = VecT<Ti>::V;
        for (auto* p : set) {
            mgp_solver* in = p->s->inner;
            const int l = p->top - d;
            LevelState& F = in->lv[l];
            LevelState& C = in->lv[l + 1];
            ProlongArgs<Ti> a{(const Ti*)u_ptr(in, l + 1), C.G, (Ti*)u_ptr(in, l), (Ti*)F.r, F.G};
            const int rows = C.G.ny * ((F.G.nz + V - 1) / V);
            push_item(items, a, (rows + kThreads - 1) / kThreads, C.G.nx);
        }
        sb.add<TProlongAdd<Ti>>(items);
    };
    std::function<void(int, const std::vector<BatchProblem*>&)> bv = [&](int d, const std::vector<BatchProblem*>& set) {
        relax(d, set);  // Vcycle<T> (include/vcycle.h:14-98) in depth terms
        if (d == 0) return;
        setup(d, set);
        bv(d - 1, set);
        prolong(d, set);
        relax(d, set);
    };
    std::function<void(int)> bff = [&](int d) {
        const auto set = members(d);
        if (d == 0) {
            relax(0, set);
            return;
        }
        relax(d, set);
        setup(d, set);
        bff(d - 1);
        prolong(d, set);
        bv(d, set);
    };
    if (b->desc.cycle == MGP_CYCLE_V) {
        std::function<void(int)> bvv = [&](int d) {
            const auto set = members(d);
            relax(d, set);
            if (d == 0) return;
            setup(d, set);
            bvv(d - 1);
            prolong(d, set);
            relax(d, set);
        };
        bvv(dmax);
    } else {
        bff(dmax);
    }
    // u += e, then the new FP64 residual, its right-hand side for the next correction and the
    // per-problem norm
    std::vector<BatchItem<UpdateArgs<double, Ti>>> ups;
    std::vector<BatchItem<RefineArgs<double, Ti>>> rrs;
    double act_points = 0.0;
    for (auto* p : act) {
        const Geom& G = p->s->lv[0].G;
        act_points += (double)G.nx * G.ny * G.nz;
    }
    for (auto* p : act) {
        mgp_solver* s = p->s;
        mgp_solver* in = s->inner;
        LevelState& L = s->lv[0];
        LevelState& I = in->lv[0];
        UpdateArgs<double, Ti> ua{(double*)u_ptr(s, 0), L.G, (const Ti*)u_ptr(in, 0), I.G.sx, I.G.sy};
        constexpr int Vd = VecT<double>::V;
        push_item(ups, ua, (L.G.ny * ((L.G.nz + Vd - 1) / Vd) + kThreads - 1) / kThreads, L.G.nx);
        RefineArgs<double, Ti> ra;
        ra.G = L.G;
        ra.u = (const double*)u_ptr(s, 0);
        ra.f = (const double*)L.f;
        ra.r = (double*)L.r;
        ra.F = faces_of<double>(s, 0);
        ra.two_h = 2.0 * L.h;
        ra.hsq = L.h * L.h;
        hsq_terms(ra.hsq, ra.inv_hsq, ra.hsq_pow2);
        ra.sxi = I.G.sx;
        ra.syi = I.G.sy;
        ra.fi = (Ti*)I.f;
        ra.ui = (Ti*)u_ptr(in, 0);
        ra.norm = b->d_norms + p->slot;
        constexpr int V = VecT<double>::V;
        const int plane = L.G.ny * ((L.G.nz + V - 1) / V);
        const int bx = (plane + kThreads - 1) / kThreads;
        const int target = std::max(1, (int)(launch_blocks * ((double)L.G.nx * L.G.ny * L.G.nz) / act_points + 0.5));
        int chunks = std::max(1, std::min((target + bx - 1) / bx, L.G.nx));
        ra.ichunk = (L.G.nx + chunks - 1) / chunks;
        chunks = (L.G.nx + ra.ichunk - 1) / ra.ichunk;
        push_item(rrs, ra, bx, chunks);
    }
    sb.add<TUpdate<Ti>>(ups);
    sb.add<TRefRes<Ti>>(rrs);
    return MGP_OK;
}

int batch_inner_dtype(const mgp_batch* b) { return b->desc.inner_dtype; }

int batch_rebuild(mgp_batch* b) {
    batch_free_schedule(b);
    // record each active problem's inner state, build (this advances it), note the post
    // state and restore: the graph launch applies the post state
    std::vector<uint64_t> pre;
    for (auto& p : b->probs) pre.push_back(p.s ? state_bits(p.s->inner) : 0);
    ScheduleBuilder sb;
    sb.sms = sm_count(b->device);
    int st = batch_inner_dtype(b) == MGP_F32 ? build_step<float>(b, sb) : build_step<double>(b, sb);
    b->post_state.clear();
    for (size_t i = 0; i < b->probs.size(); i++) {
        b->post_state.push_back(b->probs[i].s ? state_bits(b->probs[i].s->inner) : 0);
        if (b->probs[i].s) set_state_bits(b->probs[i].s->inner, pre[i]);
    }
    b->sched_state = pre;
    if (st != MGP_OK) return st;
    if (sb.bytes.size() > b->d_items_bytes) {
        if (b->d_items) cudaFree(b->d_items);
        b->d_items = nullptr;
        b->d_items_bytes = 0;
        CK(cudaMalloc(&b->d_items, sb.bytes.size()));
        b->d_items_bytes = sb.bytes.size();
    }
    if (!sb.bytes.empty())
        CK(cudaMemcpyAsync(b->d_items, sb.bytes.data(), sb.bytes.size(), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    b->launches = sb.launches;
    if (!b->launches.empty()) b->launches_last = (int64_t)b->launches.size();
    b->dirty = false;
    return MGP_OK;
}

// One step's launches issued directly on the batch stream: the steps right after the active
// set changed run this way (capturing and instantiating a graph of a few hundred launches
// costs more than launching them a few times; the host issues them while the GPU works).
constexpr int kBatchCaptureAfter = 3;
int batch_launch_direct(mgp_batch* b) {
    CK(cudaMemsetAsync(b->d_norms, 0, sizeof(unsigned long long) * b->slots, b->stream));
    for (auto& L : b->launches) L.fn((const char*)b->d_items + L.offset, L.n, L.total, L.grid, b->stream);
    CK(cudaGetLastError());
    return MGP_OK;
}

// Capture of the current schedule, replayed every step while the active set stays the same.
int batch_capture(mgp_batch* b) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    // the step's last launch max-reduces each problem's residual into its slot
    cudaError_t me = cudaMemsetAsync(b->d_norms, 0, sizeof(unsigned long long) * b->slots, b->stream);
    for (auto& L : b->launches) L.fn((const char*)b->d_items + L.offset, L.n, L.total, L.grid, b->stream);
    if (me != cudaSuccess) {
        cudaGraph_t g0 = nullptr;
        cudaStreamEndCapture(b->stream, &g0);
        if (g0) cudaGraphDestroy(g0);
        return fail(MGP_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(me));
    }
    cudaError_t le = cudaGetLastError();
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (le != cudaSuccess || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(MGP_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(le != cudaSuccess ? le : e));
    }
    cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        b->graph = nullptr;
        return fail(MGP_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(ei));
    }
    return MGP_OK;
}

BatchProblem* batch_find(mgp_batch* b, int id) {
    for (auto& p : b->probs)
        if (p.id == id && p.s) return &p;
    return nullptr;
}

// f norm and first FP64 residual of problems that have not started (their data is on the
// device now); each is its own small launch on the batch stream.
int batch_start_new(mgp_batch* b) {
    bool any = false;
    for (auto& p : b->probs) {
        if (!p.s || p.started || !p.active) continue;
        mgp_solver* s = p.s;
        std::swap(s->stream, b->stream);  // issue on the batch stream
        unsigned long long* saved = s->d_norm;
        s->d_norm = b->d_norms + p.slot;
        int st = MGP_OK;
        cudaError_t e = cudaMemsetAsync(s->d_norm, 0, 8, s->stream);
        if (e == cudaSuccess) st = norm_t<double>(s, s->lv[0].f, 0, s->d_norm);
        if (st == MGP_OK && e == cudaSuccess) e = cudaMemcpyAsync(b->h_norms + p.slot, s->d_norm, 8, cudaMemcpyDeviceToHost, s->stream);
        if (st == MGP_OK && e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (st == MGP_OK && e == cudaSuccess) {
            memcpy(&p.fnorm, b->h_norms + p.slot, 8);
            st = refine_residual(s, false);  // zeroes the inner guess, norm into the slot
        }
        if (st == MGP_OK && e == cudaSuccess) e = cudaMemcpyAsync(b->h_norms + p.slot, s->d_norm, 8, cudaMemcpyDeviceToHost, s->stream);
        if (st == MGP_OK && e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        s->d_norm = saved;
        std::swap(s->stream, b->stream);
        if (e != cudaSuccess) return fail(MGP_ERR_CUDA, "batch start: %s", cudaGetErrorString(e));
        if (st != MGP_OK) return st;
        double rn;
        memcpy(&rn, b->h_norms + p.slot, 8);
        p.rel = p.first_rel = rn / p.fnorm;
        p.started = true;
        p.iters = 0;
        any = true;
    }
    if (any) b->dirty = true;
    return MGP_OK;
}

}  // namespace

extern "C" {

int mgp_batch_create(const mgp_batch_desc* d, mgp_batch** out) {
    if (!d || !out) return fail(MGP_ERR_INVALID_ARG, "null descriptor or out pointer");
    *out = nullptr;
    if (d->inner_dtype != MGP_F32 && d->inner_dtype != MGP_F64) return fail(MGP_ERR_INVALID_ARG, "inner dtype");
    if (d->restriction != MGP_INJECTION && d->restriction != MGP_FULLWEIGHTING)
        return fail(MGP_ERR_INVALID_ARG, "unknown restriction");
    if (d->relaxation != MGP_JACOBI && d->relaxation != MGP_GAUSSSEIDEL) return fail(MGP_ERR_INVALID_ARG, "unknown relaxation");
    if (d->cycle != MGP_CYCLE_F && d->cycle != MGP_CYCLE_V) return fail(MGP_ERR_INVALID_ARG, "batch cycles are V or F");
    if (d->nsmooth < 0) return fail(MGP_ERR_INVALID_ARG, "nsmooth must be >= 0");
    if (d->max_problems < 1 || d->max_problems > (1 << 20)) return fail(MGP_ERR_INVALID_ARG, "max_problems");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(MGP_ERR_NO_DEVICE, "no CUDA device");
    if (d->device < 0 || d->device >= ndev) return fail(MGP_ERR_NO_DEVICE, "device %d not present", d->device);
    DeviceGuard guard(d->device);
    mgp_batch* b = new (std::nothrow) mgp_batch();
    if (!b) return fail(MGP_ERR_OOM, "host allocation failed");
    b->desc = *d;
    b->device = d->device;
    b->slots = (int)d->max_problems;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_norms, sizeof(unsigned long long) * b->slots);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_norms, sizeof(unsigned long long) * b->slots);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_slab, 64 * (size_t)b->slots);
    if (e == cudaSuccess) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = b->device;
        e = cudaMemPoolCreate(&b->pool, &props);
        if (e != cudaSuccess) b->pool = nullptr;
    }
    if (e == cudaSuccess) {
        uint64_t keep = UINT64_MAX;  // memory freed into the pool stays reserved for the next problem
        e = cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e != cudaSuccess) {
        if (b->d_norms) cudaFree(b->d_norms);
        if (b->h_norms) cudaFreeHost(b->h_norms);
        if (b->h_slab) cudaFreeHost(b->h_slab);
        if (b->pool) cudaMemPoolDestroy(b->pool);
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        return fail(e == cudaErrorMemoryAllocation ? MGP_ERR_OOM : MGP_ERR_CUDA, "batch set-up: %s", cudaGetErrorString(e));
    }
    *out = b;
    return MGP_OK;
}

int mgp_batch_destroy(mgp_batch* b) {
    if (!b) return MGP_OK;
    DeviceGuard guard(b->device);
    cudaStreamSynchronize(b->stream);
    batch_free_schedule(b);
    for (auto& p : b->probs)
        if (p.s) mgp_destroy(p.s);
    cudaStreamSynchronize(b->stream);  // the problems' memory is back in the pool
    if (b->pool) cudaMemPoolDestroy(b->pool);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_norms) cudaFree(b->d_norms);
    if (b->h_norms) cudaFreeHost(b->h_norms);
    if (b->h_slab) cudaFreeHost(b->h_slab);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return MGP_OK;
}

int mgp_batch_problem_bytes(const mgp_batch_desc* bd, const mgp_desc* d, int64_t* bytes) {
    if (!bd || !d || !bytes) return fail(MGP_ERR_INVALID_ARG, "null argument");
    const size_t ei = bd->inner_dtype == MGP_F32 ? 4 : 8;
    const int nbuf = bd->relaxation == MGP_JACOBI ? 2 : 1;
    int64_t total = 0;
    for (int64_t l = 0; l < d->levels; l++) {
        mgp_level_info li;
        CKS(mgp_plan_level(d, (int)l, &li));
        const int64_t al = 64 / (int64_t)ei;
        const int64_t pts = li.shape[0] * li.shape[1] * ((li.shape[2] + al - 1) / al * al);
        int64_t faces = 0;
        for (int f = 0; f < 6; f++) faces += li.face_shape[f][0] * li.face_shape[f][1] * li.face_shape[f][2];
        total += (int64_t)ei * ((nbuf + 2) * pts + faces);  // inner u (x nbuf), f, r, faces
        if (l == 0) {
            const int64_t pts8 = li.shape[0] * li.shape[1] * ((li.shape[2] + 7) / 8 * 8);
            total += 8 * ((nbuf + 2) * pts8 + faces);  // outer FP64 level 0
        }
    }
    *bytes = total + (2 << 20);
    return MGP_OK;
}

int mgp_batch_add(mgp_batch* b, const mgp_desc* problem, int* id) {
    if (!b || !problem || !id) return fail(MGP_ERR_INVALID_ARG, "null argument");
    int used = 0;
    for (auto& p : b->probs) used += p.s != nullptr;
    if (used >= b->slots) return fail(MGP_ERR_STATE, "batch is full (%d problems)", b->slots);
    mgp_desc d = *problem;
    d.dtype = MGP_F64;
    d.device = b->device;
    d.restriction = b->desc.restriction;
    d.relaxation = b->desc.relaxation;
    d.prolongation = MGP_TRILINEAR;
    d.flags = (d.flags & MGP_FLAG_STRICT_BC) | (b->desc.inner_dtype == MGP_F32 ? MGP_FLAG_REFINE_F32 : MGP_FLAG_REFINE_F64);
    // slot: lowest free
    std::vector<char> taken(b->slots, 0);
    for (auto& p : b->probs)
        if (p.s) taken[p.slot] = 1;
    int slot = 0;
    while (slot < b->slots && taken[slot]) slot++;
    mgp_solver* s = nullptr;
    const CreateCtx ctx{b->stream, b->pool, b->h_slab + 8 * (size_t)slot};
    CKS(create_solver(&d, &s, &ctx));
    BatchProblem p;
    p.id = b->next_id++;
    p.s = s;
    p.top = (int)d.levels - 1;
    p.slot = slot;
    // reuse a retired entry's place
    bool placed = false;
    for (auto& q : b->probs)
        if (!q.s) {
            q = p;
            placed = true;
            break;
        }
    if (!placed) b->probs.push_back(p);
    b->dirty = true;
    *id = p.id;
    return MGP_OK;
}

int mgp_batch_problem(mgp_batch* b, int id, mgp_solver** s) {
    if (!b || !s) return fail(MGP_ERR_INVALID_ARG, "null argument");
    BatchProblem* p = batch_find(b, id);
    if (!p) return fail(MGP_ERR_INVALID_ARG, "no problem %d in the batch", id);
    *s = p->s;
    return MGP_OK;
}

int mgp_batch_remove(mgp_batch* b, int id) {
    if (!b) return fail(MGP_ERR_INVALID_ARG, "null batch");
    BatchProblem* p = batch_find(b, id);
    if (!p) return fail(MGP_ERR_INVALID_ARG, "no problem %d in the batch", id);
    DeviceGuard guard(b->device);
    cudaStreamSynchronize(b->stream);
    batch_free_schedule(b);  // the graph refers to this problem's buffers
    mgp_destroy(p->s);
    p->s = nullptr;
    p->active = false;
    b->dirty = true;
    return MGP_OK;
}

int mgp_batch_set_active(mgp_batch* b, int id, int active) {
    if (!b) return fail(MGP_ERR_INVALID_ARG, "null batch");
    BatchProblem* p = batch_find(b, id);
    if (!p) return fail(MGP_ERR_INVALID_ARG, "no problem %d in the batch", id);
    if (p->active != (active != 0)) b->dirty = true;
    p->active = active != 0;
    return MGP_OK;
}

int mgp_batch_step(mgp_batch* b, int* n_active) {
    if (!b) return fail(MGP_ERR_INVALID_ARG, "null batch");
    DeviceGuard guard(b->device);
    CKS(batch_start_new(b));
    std::vector<uint64_t> cur;
    for (auto& p : b->probs) cur.push_back(p.s ? state_bits(p.s->inner) : 0);
    const bool changed = b->dirty || cur != b->sched_state;
    if (changed) {
        CKS(batch_rebuild(b));  // schedule only
        b->stable_steps = 0;
    } else if (!b->graph && !b->launches.empty() && b->stable_steps >= kBatchCaptureAfter) {
        CKS(batch_capture(b));  // the set has held for a while: replay it as a graph
    }
    b->stable_steps++;
    int n = 0;
    for (auto& p : b->probs) n += (p.s && p.active && p.started);
    if (n_active) *n_active = n;
    if (!n || b->launches.empty()) return MGP_OK;
    if (b->graph) CK(cudaGraphLaunch(b->graph, b->stream));
    else CKS(batch_launch_direct(b));
    b->launches_total += (int64_t)b->launches.size();
    CK(cudaMemcpyAsync(b->h_norms, b->d_norms, sizeof(unsigned long long) * b->slots, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    for (size_t i = 0; i < b->probs.size(); i++) {
        BatchProblem& p = b->probs[i];
        if (!p.s) continue;
        set_state_bits(p.s->inner, b->post_state[i]);
        if (!p.active || !p.started) continue;
        double rn;
        memcpy(&rn, b->h_norms + p.slot, 8);
        p.rel = rn / p.fnorm;
        p.iters++;
    }
    b->sched_state.clear();
    for (auto& p : b->probs) b->sched_state.push_back(p.s ? state_bits(p.s->inner) : 0);
    return MGP_OK;
}

int mgp_batch_restart(mgp_batch* b, int id) {
    if (!b) return fail(MGP_ERR_INVALID_ARG, "null batch");
    BatchProblem* p = batch_find(b, id);
    if (!p) return fail(MGP_ERR_INVALID_ARG, "no problem %d in the batch", id);
    p->started = false;
    p->active = true;
    p->iters = 0;
    b->dirty = true;
    return MGP_OK;
}

int mgp_batch_status(mgp_batch* b, int id, mgp_stats* out) {
    if (!b || !out) return fail(MGP_ERR_INVALID_ARG, "null argument");
    BatchProblem* p = batch_find(b, id);
    if (!p) return fail(MGP_ERR_INVALID_ARG, "no problem %d in the batch", id);
    memset(out, 0, sizeof(*out));
    out->rel_res = p->rel;
    out->iterations = (double)p->iters;
    out->cycles_run = p->iters;
    out->first_rel_res = p->first_rel;
    return MGP_OK;
}

int mgp_batch_solve(mgp_batch* b, double tol, int64_t maxiter, int64_t* steps) {
    if (!b) return fail(MGP_ERR_INVALID_ARG, "null batch");
    int64_t k = 0;
    CKS(batch_start_new(b));
    for (auto& p : b->probs)
        if (p.s && p.active && p.started && p.rel < tol) CKS(mgp_batch_set_active(b, p.id, 0));
    while (k < maxiter) {
        int n = 0;
        CKS(mgp_batch_step(b, &n));
        if (!n) break;
        k++;
        for (auto& p : b->probs)
            if (p.s && p.active && p.started && p.rel < tol) CKS(mgp_batch_set_active(b, p.id, 0));
    }
    // the user-visible FP64 residual of every problem
    DeviceGuard guard(b->device);
    for (auto& p : b->probs)
        if (p.s) {
            std::swap(p.s->stream, b->stream);
            int st = refine_residual(p.s, true);
            std::swap(p.s->stream, b->stream);
            CKS(st);
        }
    CK(cudaStreamSynchronize(b->stream));
    if (steps) *steps = k;
    return MGP_OK;
}

int mgp_batch_kernel_launches(const mgp_batch* b, int64_t* per_step) {
    if (!b || !per_step) return fail(MGP_ERR_INVALID_ARG, "null argument");
    *per_step = b->launches.empty() ? b->launches_last : (int64_t)b->launches.size();
    return MGP_OK;
}

int mgp_batch_reserve(mgp_batch* b, size_t bytes) {
    if (!b) return fail(MGP_ERR_INVALID_ARG, "null batch");
    if (!bytes) return MGP_OK;
    DeviceGuard guard(b->device);
    void* p = nullptr;
    const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, b->pool, b->stream);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? MGP_ERR_OOM : MGP_ERR_CUDA, "reserving %zu bytes: %s", bytes,
                    cudaGetErrorString(e));
    CK(cudaFreeAsync(p, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return MGP_OK;
}

int mgp_batch_mem_info(mgp_batch* b, size_t* free_bytes, size_t* total_bytes) {
    if (!b || !free_bytes || !total_bytes) return fail(MGP_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(b->device);
    CK(cudaMemGetInfo(free_bytes, total_bytes));
    uint64_t reserved = 0, used = 0;
    CK(cudaMemPoolGetAttribute(b->pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    CK(cudaMemPoolGetAttribute(b->pool, cudaMemPoolAttrUsedMemCurrent, &used));
    if (reserved > used) *free_bytes += (size_t)(reserved - used);
    return MGP_OK;
}

}  // extern "C"
