// mgp_stencil_tma.cuh -- the 7-point stencil sweeps of large levels, fed by TMA.
//
// Same operations and arithmetic as stencil_tile (Jacobi, red-black / column-ordered
// Gauss-Seidel, residual with optional max-norm), different data movement.  A CTA owns a tile
// of TJ rows (j) x BK points (k) and marches it along i.  Planes of u (the tile plus one halo
// row on each side in j and HK = 16 bytes of halo on each side in k) and of f (the tile only)
// are brought into shared-memory rings by cp.async.bulk.tensor, issued by one thread up to
// three planes ahead of the plane being computed; every neighbour of a point is then a
// shared-memory read, so the stencil's in-plane and out-of-plane reuse never goes back to
// L1/L2.  A __syncthreads per plane hands the slot of plane i-1 back to the producer.
//
// Work split: the (tile, plane) pairs of the level are cut into gridDim.x equal contiguous
// ranges, one per CTA (one wave of resident CTAs, no tail); a range is at most a few
// (tile, i-chunk) segments.  Column-ordered Gauss-Seidel needs each column swept in i order
// by one CTA, so there every CTA takes one whole tile.
//
// Launched in ordinary stream order, never as a programmatic dependent: a sweep launched early
// behind a running grid read stale data on B200 (reproduced with a TMA sweep following
// another TMA sweep of a different level geometry; it went away once that launch waited for
// the previous grid to complete).
//
// Waits on the ring barriers are bounded: a wait that runs out sets *err and the CTA stops
// computing; thread 0 then waits (bounded again) for the copies it issued before the CTA
// exits, so that no copy lands in shared memory the CTA no longer owns.
#include <cuda.h>

namespace mgp {

constexpr int kTmaTJ = 4;        // rows per tile
constexpr int kTmaRingU = 5;     // u planes in shared memory: i-1, i, i+1 and two in flight
constexpr int kTmaRingF = 4;     // f planes: i and three in flight
constexpr int kTmaMaxThreads = 288;

struct TmaTiling {
    int BK;              // k points per tile (multiple of V and of HK)
    int ntj, ntk;        // tiles in j and k
    int nvec;            // threads per row = BK / V
    int slot_u, slot_f;  // ring slot sizes in bytes (multiples of 128)
    long long work;      // ntj * ntk * nx (tile-planes)
    int whole_tiles;     // 1: every CTA sweeps one whole tile (column-ordered Gauss-Seidel)
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false after 2^22 polls (each try_wait suspends the thread for a while).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    for (unsigned n = 0; n < (1u << 22); n++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <typename T>
__host__ __device__ constexpr int tma_hk() {
    return 16 / (int)sizeof(T);
}

template <typename T, int OP, bool NORM>
__global__ void __launch_bounds__(kTmaMaxThreads, 1)
    k_stencil_tma(const __grid_constant__ CUtensorMap map_u, const __grid_constant__ CUtensorMap map_f,
                  StencilArgs<T> a, TmaTiling tl, int* err) {
    constexpr int V = VecT<T>::V;
    constexpr int HK = tma_hk<T>();
    constexpr int TJ = kTmaTJ;
    extern __shared__ unsigned char smem_raw[];
    __shared__ unsigned long long bar_u[kTmaRingU], bar_f[kTmaRingF];
    const Geom& G = a.G;
    const int BK = tl.BK, W = BK + 2 * HK;  // u slot row length (elements)
    const int nvec = tl.nvec;
    const int jr = threadIdx.x / nvec, kv = threadIdx.x - jr * nvec;
    unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    T* ring_u = reinterpret_cast<T*>(smem);
    T* ring_f = reinterpret_cast<T*>(smem + (size_t)kTmaRingU * tl.slot_u);
    const int su = tl.slot_u / (int)sizeof(T), sf = tl.slot_f / (int)sizeof(T);
    const unsigned bytes_u = (unsigned)((TJ + 2) * W * sizeof(T)), bytes_f = (unsigned)(TJ * BK * sizeof(T));
    if (threadIdx.x == 0) {
        for (int s = 0; s < kTmaRingU; s++) mbar_init(&bar_u[s], 1);
        for (int s = 0; s < kTmaRingF; s++) mbar_init(&bar_f[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    unsigned ph_u = 0u, ph_f = 0u;      // parity of each slot's next completion (bit per slot)
    unsigned pend_u = 0u, pend_f = 0u;  // thread 0: slots with a copy issued and not yet waited
    unsigned long long mx = 0ull;
    const long long per = (tl.work + gridDim.x - 1) / gridDim.x;
    long long w = tl.whole_tiles ? (long long)blockIdx.x * G.nx : (long long)blockIdx.x * per;
    const long long w_end = tl.whole_tiles ? w + G.nx : min(tl.work, w + per);
    const T two_h = a.two_h, m2h = -two_h;
    const unsigned full = (1u << V) - 1u;
    bool failed = false;
    while (w < w_end) {
        const int tile = (int)(w / G.nx);
        const int ia = (int)(w - (long long)tile * G.nx);
        const int ib = (int)min((long long)G.nx, ia + (w_end - w));
        w += ib - ia;
        const int tj = tile % tl.ntj, tk = tile / tl.ntj;
        const int j0 = tj * TJ, k0 = tk * BK;
        // u planes [pu0, pu1) = ia-1 .. ib inside the level; f planes [ia, ib).  Plane p uses
        // slot p % ring; each plane is issued once and waited once.
        const int pu0 = max(ia - 1, 0), pu1 = min(ib + 1, G.nx);
        if (threadIdx.x == 0) {
            for (int p = pu0; p < min(pu1, pu0 + kTmaRingU); p++) {
                const int sl = p % kTmaRingU;
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                mbar_expect_tx(&bar_u[sl], bytes_u);
                tma_load_3d(ring_u + (size_t)sl * su, &map_u, k0 - HK, j0 - 1, p, &bar_u[sl]);
                pend_u |= 1u << sl;
            }
            for (int p = ia; p < min(ib, ia + kTmaRingF); p++) {
                const int sl = p % kTmaRingF;
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                mbar_expect_tx(&bar_f[sl], bytes_f);
                tma_load_3d(ring_f + (size_t)sl * sf, &map_f, k0, j0, p, &bar_f[sl]);
                pend_f |= 1u << sl;
            }
        }
        bool ok = true;
        for (int p = pu0; p <= ia && ok; p++) {
            const int sl = p % kTmaRingU;
            ok = mbar_wait(&bar_u[sl], (ph_u >> sl) & 1u);
            if (ok) {
                ph_u ^= 1u << sl;
                pend_u &= ~(1u << sl);
            }
        }
        // this thread's point vector of the tile
        const int j = j0 + jr, kb = k0 + kv * V;
        const bool mine = j < G.ny && kb < G.nz;
        const bool jin = j >= G.y0 && j < G.y1;
        unsigned ins = 0u, inr = 0u;
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int k = kb + e;
            if (mine && k < G.nz) ins |= 1u << e;
            if (mine && k < G.nz && jin && k >= G.z0 && k < G.z1) inr |= 1u << e;
        }
        const size_t row = (size_t)(jr + 1) * W + HK + kv * V;  // this vector in a u slot
        T vmo[V];  // u(i-1) as it was before this sweep (east ghost mirror)
        if (ins) {
            const T* Um0 = ia > 0 ? ring_u + (size_t)((ia - 1) % kTmaRingU) * su + row : nullptr;
#pragma unroll
            for (int e = 0; e < V; e++) vmo[e] = Um0 ? Um0[e] : T(0);
        }
        for (int i = ia; i < ib; i++) {
            if (ok && i + 1 < pu1) {
                const int sl = (i + 1) % kTmaRingU;
                ok = mbar_wait(&bar_u[sl], (ph_u >> sl) & 1u);
                if (ok) {
                    ph_u ^= 1u << sl;
                    pend_u &= ~(1u << sl);
                }
            }
            if (ok) {
                const int sl = i % kTmaRingF;
                ok = mbar_wait(&bar_f[sl], (ph_f >> sl) & 1u);
                if (ok) {
                    ph_f ^= 1u << sl;
                    pend_f &= ~(1u << sl);
                }
            }
            if (!ok) atomicExch(err, 1);
            const T* Uc = ring_u + (size_t)(i % kTmaRingU) * su + row;
            const T* Um = i > 0 ? ring_u + (size_t)((i - 1) % kTmaRingU) * su + row : nullptr;
            const T* Up = i + 1 < G.nx ? ring_u + (size_t)((i + 1) % kTmaRingU) * su + row : nullptr;
            const T* Fc = ring_f + (size_t)(i % kTmaRingF) * sf + (size_t)jr * BK + kv * V;
            const bool iin = i >= G.x0 && i < G.x1;
            if (ok && ins) {
                if (NORM) {
                    // r outside the relaxation bounds keeps its value and counts in the norm
                    const unsigned m = iin ? (ins & ~inr) : ins;
                    const T* rp = a.dst + (long long)i * G.sx + (long long)j * G.sy + kb;
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if ((m >> e) & 1u) mx = max(mx, abs_bits(rp[e]));
                }
                unsigned act = iin ? inr : 0u;
                if (OP == OP_GS || OP == OP_GS_COLUMN) {
                    const int base = (OP == OP_GS ? i : 0) + j + kb + G.poff;
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if (((base + e) & 1) != a.colour) act &= ~(1u << e);
                }
                T vc[V];
                lds_v(vc, Uc);
                if (act) {
                    T vm[V], vp[V], ym[V], yp[V], fc[V];
                    if (i > 0) {
                        lds_v(vm, Um);
                    } else {  // west ghost  -2h*gW + u(1)
#pragma unroll
                        for (int e = 0; e < V; e++)
                            vm[e] = ((ins >> e) & 1u) ? m2h * ldg(a.F.g[F_WEST] + (long long)j * G.nz + kb + e) + Up[e]
                                                      : T(0);
                    }
                    if (i + 1 < G.nx) {
                        lds_v(vp, Up);
                    } else {  // east ghost  2h*gE + u(nx-2), from before this sweep
#pragma unroll
                        for (int e = 0; e < V; e++)
                            vp[e] = ((ins >> e) & 1u) ? two_h * ldg(a.F.g[F_EAST] + (long long)j * G.nz + kb + e) + vmo[e]
                                                      : T(0);
                    }
                    if (j > 0) {
                        lds_v(ym, Uc - W);
                    } else {  // south ghost  -2h*gS + u(j=1)
#pragma unroll
                        for (int e = 0; e < V; e++)
                            ym[e] = ((ins >> e) & 1u) ? m2h * ldg(a.F.g[F_SOUTH] + (long long)i * G.nz + kb + e) + Uc[W + e]
                                                      : T(0);
                    }
                    if (j < G.ny - 1) {
                        lds_v(yp, Uc + W);
                    } else {  // north ghost  2h*gN + u(j=ny-2)
#pragma unroll
                        for (int e = 0; e < V; e++)
                            yp[e] = ((ins >> e) & 1u) ? two_h * ldg(a.F.g[F_NORTH] + (long long)i * G.nz + kb + e) + Uc[e - W]
                                                      : T(0);
                    }
                    lds_v(fc, Fc);
                    const T left = Uc[-1], right = Uc[V];
                    T cur[V];
#pragma unroll
                    for (int e = 0; e < V; e++) {
                        cur[e] = vc[e];
                        if (!((act >> e) & 1u)) continue;
                        const int k = kb + e;
                        const T below = e > 0 ? vc[e - 1] : left;       // u(k-1)
                        const T above = e < V - 1 ? vc[e + 1] : right;  // u(k+1)
                        T zm, zp;
                        if (k > 0) zm = below;
                        else zm = m2h * ldg(a.F.g[F_BOTTOM] + (long long)i * G.ny + j) + vc[1];  // -2h*gB + u(1)
                        if (k < G.nz - 1) zp = above;
                        else zp = two_h * ldg(a.F.g[F_TOP] + (long long)i * G.ny + j) + below;  // 2h*gT + u(nz-2)
                        const T sum = vm[e] + vp[e] + ym[e] + yp[e] + zm + zp;
                        if (OP == OP_RESIDUAL) {
                            const T r = residual_pt(fc[e], sum, vc[e], a.hsq, a.inv_hsq, a.hsq_pow2);
                            cur[e] = r;
                            if (NORM) mx = max(mx, abs_bits(r));
                        } else {
                            // jacobi.h:59-61 / gaussseidel.h:43-45
                            cur[e] = a.one_omega * vc[e] + a.omega_sixth * (sum - a.hsq * fc[e]);
                        }
                    }
                    T* out = a.dst + (long long)i * G.sx + (long long)j * G.sy + kb;
                    const unsigned wm = (OP == OP_GS || OP == OP_GS_COLUMN) ? ins : act;
                    if (wm == full) {
                        stv(out, cur);
                    } else {
#pragma unroll
                        for (int e = 0; e < V; e++)
                            if ((wm >> e) & 1u) out[e] = cur[e];
                    }
                    if (OP == OP_GS_COLUMN) {
                        // in column order the next plane's west neighbour is this plane's new value
                        T* uw = const_cast<T*>(Uc);
#pragma unroll
                        for (int e = 0; e < V; e++) uw[e] = cur[e];
                    }
                }
#pragma unroll
                for (int e = 0; e < V; e++) vmo[e] = vc[e];
            }
            // the column-order write-backs into the ring are generic-proxy writes to a slot that
            // a later copy (async proxy) refills: each writer orders them before the barrier
            if (OP == OP_GS_COLUMN) asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            // plane i-1's u slot and plane i's f slot are free again; stop if any wait failed
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            if (threadIdx.x == 0) {
                const int pn = i - 1 + kTmaRingU;  // next u plane, into plane (i-1)'s slot
                if (i - 1 >= pu0 && pn < pu1) {
                    const int sl = pn % kTmaRingU;
                    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                    mbar_expect_tx(&bar_u[sl], bytes_u);
                    tma_load_3d(ring_u + (size_t)sl * su, &map_u, k0 - HK, j0 - 1, pn, &bar_u[sl]);
                    pend_u |= 1u << sl;
                }
                const int qn = i + kTmaRingF;      // next f plane, into plane i's slot
                if (qn < ib) {
                    const int sl = qn % kTmaRingF;
                    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                    mbar_expect_tx(&bar_f[sl], bytes_f);
                    tma_load_3d(ring_f + (size_t)sl * sf, &map_f, k0, j0, qn, &bar_f[sl]);
                    pend_f |= 1u << sl;
                }
            }
        }
        if (failed) break;
        __syncthreads();  // the next segment's copies overwrite slots this one read
    }
    if (failed && threadIdx.x == 0) {
        // let the copies already issued land before the CTA's shared memory is released
        for (int s = 0; s < kTmaRingU; s++)
            if ((pend_u >> s) & 1u) mbar_wait(&bar_u[s], (ph_u >> s) & 1u);
        for (int s = 0; s < kTmaRingF; s++)
            if ((pend_f >> s) & 1u) mbar_wait(&bar_f[s], (ph_f >> s) & 1u);
    }
    if (NORM) block_max_to(mx, a.norm);
}

}  // namespace mgp
