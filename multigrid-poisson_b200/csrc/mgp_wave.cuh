// mgp_wave.cuh -- stencil passes of large levels, chained in one TMA-fed march.
//
// Relaxation<T>::relax with Jacobi (include/relaxation.h:19-94, include/jacobi.h:39-82) reads
// u_prev and f and writes u once per sweep, and residual<T> (include/residual.h:17-81) reads u
// and f and writes r.  On a large level each of those is one pass over HBM.  This kernel makes
// up to three of them -- "stages" -- in a single march along i:
//
//     NJ Jacobi sweeps (0, 1 or 2), then optionally the residual of their result (RES):
//       (J)  (J,J)  (R)  (J,R)  (J,J,R)
//
// At step t stage 1 computes plane t, stage 2 plane t-1 and stage 3 plane t-2, each from the
// previous stage's output, with every value and every operation as the reference makes them:
// the same expressions in the same order, the Neumann ghost formula (sign*2h)*g + u[mirror]
// (include/neumann.h:63-131) applied to the field that stage reads, and the reference's values
// at the points a sweep leaves alone.  Sweep 1 writes into u_prev's buffer (swap_u,
// include/domain.h:311-316), so its output at unrelaxed points is u_prev's own value; sweep 2
// writes into u's buffer, so its output there is u's own value.
//
// Buffers.  A = u (u0), read through TMA.  B = u_prev.  One sweep (NJ = 1): u1 is written into B
// at relaxed points (B becomes u, as in the reference).  Two sweeps (NJ = 2): u2 goes to a third
// buffer C -- writing it over A is impossible while other CTAs still read A's halo rows -- at
// every shape point (u2 where relaxed, A's own values elsewhere), and C becomes u; with WU1, u1
// is also written into B at relaxed points (otherwise B's relaxed points are left stale, which
// the engine allows only where a later sweep rewrites them before anything reads them).
// RES: r at relaxed points; RES == 2 also reduces max |r| over the tile's points into *norm,
// including the stored r at unrelaxed points (infinity_norm runs over the whole shape,
// include/devicearray.h:211-237).
//
// Data movement.  A CTA owns TJ rows (j) x every k of the level, and a chunk of planes
// [ia, ib).  Its threads cover rows = TJ + 2(M-1) rows (stage s is computed on the middle
// TJ + 2(M-s) of them; the outer ones are halo rows that the later stages need as neighbours),
// one 16-byte vector of k points each.  One thread issues cp.async.bulk.tensor copies of u0
// planes (rows + 2 rows; with them, where a second stage reads sweep 1's output, u_prev's
// values on the Dirichlet boundary lines of the tile: the k = 0 and k = nz-1 columns and the
// j = 0 and j = ny-1 rows) and of f planes into shared-memory rings, two planes ahead of use
// (the f ring also keeps the M-1 planes the later stages still read), plus L2 prefetches of
// the same data l2a planes further on, so the DRAM stream runs well ahead of the
// compute while the rings stay small.  The output of every stage except the last goes into a
// two-plane shared buffer, where the next stage reads it: in-plane neighbours and the own
// column of its plane; the own column of the plane after comes from the stage just run (a
// register) and that of the plane before is read at the start of the step, before the earlier
// stage overwrites its parity.  Only u0(t-1) is carried from step to step in registers.
// Thread 0 waits for the next step's planes before the step's __syncthreads, so no other
// thread polls a ring barrier for long.  The grid lists the tiles of a chunk next to each other,
// so the CTAs that share halo rows march the same planes at the same time and the halo rows
// come from L2, not DRAM.  Global loads inside a step remain only for rare data: Neumann face
// values on the faces' lines and u_prev on a Dirichlet x plane.
//
// Waits on the ring barriers are bounded: a wait that runs out sets *err and every thread stops
// computing; thread 0 then waits (bounded again) for the copies it issued before the CTA exits,
// so that no copy lands in shared memory the CTA no longer owns.
#pragma once
#include <cuda.h>

#include <type_traits>

namespace mgp {

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
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false after `polls` polls.  The first poll does not block (test_wait), the
// others may suspend the thread for a while (try_wait); a bound of one poll thus fails on any
// copy still in flight.
constexpr unsigned kWaitPolls = 1u << 22;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned polls = kWaitPolls) {
    if (polls == 0) return false;
    if (mbar_test_wait(bar, parity)) return true;
    for (unsigned n = 1; n < polls; n++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

constexpr int kWaveMaxRing = 10;   // ring slots (u0 ring; the f ring has up to two more)
constexpr int kWaveMaxThreads = 608;  // consumers; with the producer, at most 5 warps per SM quadrant (96 registers)
constexpr int kWaveMaxWidth = 256; // elements in one row of a TMA box

// Tiling of a level for an M-stage pass (chosen on the host).  Byte sizes; every sub-buffer
// starts on a 128-byte boundary.
struct WaveTile {
    bool ok = false;
    int TJ = 0, rows = 0, nvec = 0, P = 0;
    int tiles_j = 0, ci = 0, chunks = 0;
    int slot_u = 0, slot_f = 0, slot_w = 0;  // u0 ring slot (with u_prev's boundary lines), f slot, work plane
    int b_klo = 0, b_khi = 0, b_jlo = 0, b_jhi = 0;  // offsets of u_prev's boundary lines in a u0 slot
    int kl = 0;                              // first k of the box holding k = nz-1 (a multiple of V)
    int ru = 0;                              // u0 ring slots: planes t, t+1 in use, ru-2 in flight
    int fa = 0;                              // f planes in flight beyond t (the f ring holds M + fa)
    int l2a = 0;                             // L2 prefetch distance beyond a plane's ring copy (planes)
    int l2mode = 0;                          // 0: none, 1: the copy's box, 2: the contiguous rows holding it
    size_t smem = 0;                         // dynamic shared memory bytes
};

template <typename T>
struct WaveArgs {
    Geom G;
    const T* A;  // u0 (the level's u)
    T* B;        // u_prev
    T* C;        // two sweeps: u2's destination
    T* r;        // residual
    const T* f;
    Faces<T> F;
    T two_h, hsq, one_omega, omega_sixth, inv_hsq;
    int hsq_pow2;
    WaveTile t;  // tiling (blockIdx.x = chunk * tiles_j + tile, blockDim.x = rows * nvec)
    unsigned long long* norm;
    int* err;
    unsigned wait_polls;  // bound of the consumers' waits for a copy (the producer's waits keep kWaitPolls)
};

__device__ __forceinline__ void tma_prefetch_l2_3d(const CUtensorMap* map, int x, int y, int z) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];\n" ::"l"(
                     reinterpret_cast<unsigned long long>(map)),
                 "r"(x), "r"(y), "r"(z)
                 : "memory");
}
__device__ __forceinline__ void bulk_prefetch_l2(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_3d_s(unsigned dst, const CUtensorMap* map, int x, int y, int z,
                                              unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(dst),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Shared-memory vectors and scalars at 32-bit shared addresses.
__device__ __forceinline__ void sld(double (&d)[2], unsigned a) {
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n" : "=d"(d[0]), "=d"(d[1]) : "r"(a));
}
__device__ __forceinline__ void sld(float (&d)[4], unsigned a) {
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n" : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3]) : "r"(a));
}
__device__ __forceinline__ void sld(float (&d)[2], unsigned a) {
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];\n" : "=f"(d[0]), "=f"(d[1]) : "r"(a));
}
__device__ __forceinline__ void sld1(double& v, unsigned a) { asm volatile("ld.shared.f64 %0, [%1];\n" : "=d"(v) : "r"(a)); }
__device__ __forceinline__ void sld1(float& v, unsigned a) { asm volatile("ld.shared.f32 %0, [%1];\n" : "=f"(v) : "r"(a)); }
__device__ __forceinline__ void sst(unsigned a, const double (&d)[2]) {
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};\n" ::"r"(a), "d"(d[0]), "d"(d[1]) : "memory");
}
__device__ __forceinline__ void sst(unsigned a, const float (&d)[2]) {
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};\n" ::"r"(a), "f"(d[0]), "f"(d[1]) : "memory");
}
__device__ __forceinline__ void sst(unsigned a, const float (&d)[4]) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"r"(a), "f"(d[0]), "f"(d[1]), "f"(d[2]), "f"(d[3])
                 : "memory");
}

// The residual f - (sum - 6u)/h^2 of residual_pt where h^2 is a power of two (x/h^2 and
// x*(1/h^2) round identically); the engine fuses the residual only on such levels.
__device__ __forceinline__ double resid_mul(double fv, double sum, double uc, double inv_hsq) {
    return fv - (sum - 6.0 * uc) * inv_hsq;
}
__device__ __forceinline__ float resid_mul(float fv, float sum, float uc, float inv_hsq) {
    const double t = (double)sum - 6.0 * (double)uc;
    return (float)((double)fv - t * (double)inv_hsq);
}

// One stencil stage at the point vector (i, j, kb) of the field it reads: Jacobi
// (jacobi.h:59-61) or, with RESID, the residual (residual.h:70-72).  c, xm, xp: the field at
// (i, j), (i-1, j), (i+1, j), own column; W: shared address of the field's plane at (j, kb),
// row pitch PB bytes (rows j-1 and j+1 at W -/+ PB; the elements just before and after the
// vector are readable, the buffers being padded).  Elements outside `act` (the relaxed points)
// keep c; a ghost is formed only at a relaxed point, i.e. on a Neumann face.
template <typename T, int V, bool RESID>
__device__ __forceinline__ void wave_point(T (&out)[V], const T (&c)[V], const T (&xm0)[V], const T (&xp0)[V],
                                           unsigned W, unsigned PB, const T (&fv)[V], unsigned act, int i, int j,
                                           int kb, const WaveArgs<T>& a) {
    const Geom& G = a.G;
    const T two_h = a.two_h, m2h = -a.two_h;
    T xm[V], xp[V], ym[V], yp[V], left, right;
    sld(ym, W - PB);
    sld(yp, W + PB);
    sld1(left, W - (unsigned)sizeof(T));
    sld1(right, W + (unsigned)(V * sizeof(T)));
#pragma unroll
    for (int e = 0; e < V; e++) {
        xm[e] = xm0[e];
        xp[e] = xp0[e];
    }
    if (act) {
        // Neumann ghosts on the lines of the faces (rare threads and planes)
        if (i == 0) {  // west ghost  -2h*gW + u(1)
            const T* g = a.F.g[F_WEST] + (long long)j * G.nz + kb;
#pragma unroll
            for (int e = 0; e < V; e++)
                if ((act >> e) & 1u) xm[e] = m2h * ldg(g + e) + xp0[e];
        }
        if (i == G.nx - 1) {  // east ghost  2h*gE + u(nx-2)
            const T* g = a.F.g[F_EAST] + (long long)j * G.nz + kb;
#pragma unroll
            for (int e = 0; e < V; e++)
                if ((act >> e) & 1u) xp[e] = two_h * ldg(g + e) + xm0[e];
        }
        if (j == 0) {  // south ghost  -2h*gS + u(j=1)
            const T* g = a.F.g[F_SOUTH] + (long long)i * G.nz + kb;
#pragma unroll
            for (int e = 0; e < V; e++)
                if ((act >> e) & 1u) ym[e] = m2h * ldg(g + e) + yp[e];
        }
        if (j == G.ny - 1) {  // north ghost  2h*gN + u(j=ny-2)
            const T* g = a.F.g[F_NORTH] + (long long)i * G.nz + kb;
#pragma unroll
            for (int e = 0; e < V; e++)
                if ((act >> e) & 1u) yp[e] = two_h * ldg(g + e) + ym[e];
        }
    }
    T zlo = left, zhi = right;  // u(kb-1), u(kb+V)
    if (kb == 0 && (act & 1u)) zlo = m2h * ldg(a.F.g[F_BOTTOM] + (long long)i * G.ny + j) + c[1];  // -2h*gB + u(1)
    const int et = G.nz - 1 - kb;  // the element holding k = nz-1, if this vector holds it
    T gt = T(0);
    if (et < V && ((act >> et) & 1u)) gt = two_h * ldg(a.F.g[F_TOP] + (long long)i * G.ny + j);
#pragma unroll
    for (int e = 0; e < V; e++) {
        const T zm = e > 0 ? c[e - 1] : zlo;
        T zp = e < V - 1 ? c[e + 1] : zhi;
        if (e == et) zp = gt + zm;  // 2h*gT + u(nz-2)
        const T sum = xm[e] + xp[e] + ym[e] + yp[e] + zm + zp;
        T v;
        if (RESID) v = resid_mul(fv[e], sum, c[e], a.inv_hsq);
        else v = a.one_omega * c[e] + a.omega_sixth * (sum - a.hsq * fv[e]);
        out[e] = ((act >> e) & 1u) ? v : c[e];
    }
}

// The same stage at a vector whose points are all relaxed and none on a face line: no ghosts,
// no masks (interior k-vectors of interior rows on interior planes).
template <typename T, int V, bool RESID>
__device__ __forceinline__ void wave_fast(T (&out)[V], const T (&c)[V], const T (&xm)[V], const T (&xp)[V],
                                          unsigned W, unsigned PB, const T (&fv)[V], const WaveArgs<T>& a) {
    T ym[V], yp[V], left, right;
    sld(ym, W - PB);
    sld(yp, W + PB);
    sld1(left, W - (unsigned)sizeof(T));
    sld1(right, W + (unsigned)(V * sizeof(T)));
#pragma unroll
    for (int e = 0; e < V; e++) {
        const T zm = e > 0 ? c[e - 1] : left;
        const T zp = e < V - 1 ? c[e + 1] : right;
        const T sum = xm[e] + xp[e] + ym[e] + yp[e] + zm + zp;
        if (RESID) out[e] = resid_mul(fv[e], sum, c[e], a.inv_hsq);
        else out[e] = a.one_omega * c[e] + a.omega_sixth * (sum - a.hsq * fv[e]);
    }
}

// Store the elements `m` of v at p (one 16-byte store when all V are stored).
template <typename T, int V>
__device__ __forceinline__ void st_masked(T* p, const T (&v)[V], unsigned m) {
    if (m == (1u << V) - 1u) {
        stv(p, v);
    } else {
#pragma unroll
        for (int e = 0; e < V; e++)
            if ((m >> e) & 1u) p[e] = v[e];
    }
}

template <typename T, int V>
__device__ __forceinline__ void norm_all(unsigned long long& mx, const T (&out)[V]) {
#pragma unroll
    for (int e = 0; e < V; e++) mx = max(mx, abs_bits(out[e]));
}

// Max-norm share of the computed r at the relaxed elements `act`.
template <typename T, int V>
__device__ __forceinline__ void norm_act(unsigned long long& mx, const T (&out)[V], unsigned act) {
#pragma unroll
    for (int e = 0; e < V; e++)
        if ((act >> e) & 1u) mx = max(mx, abs_bits(out[e]));
}

// A ring position: slot index and the parity of its next barrier phase.
struct RingPos {
    int slot;
    unsigned par;
    __device__ __forceinline__ void next(int n) {
        if (++slot == n) {
            slot = 0;
            par ^= 1u;
        }
    }
};

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait; a wait that runs out records the failure in *err.
__device__ __forceinline__ bool wave_wait(unsigned long long* bar, unsigned par, int* err,
                                          unsigned polls = kWaitPolls) {
    if (mbar_wait(bar, par, polls)) return true;
    atomicExch(err, 1);
    return false;
}

template <typename T, int NJ, int RES, bool WU1>
__global__ void __launch_bounds__(kWaveMaxThreads + 32, 1)
    k_wave(const __grid_constant__ CUtensorMap map_u, const __grid_constant__ CUtensorMap map_f,
           const __grid_constant__ CUtensorMap map_bk, const __grid_constant__ CUtensorMap map_bj, WaveArgs<T> a) {
    constexpr int V = VecT<T>::V;
    constexpr unsigned ES = sizeof(T);
    constexpr int M = NJ + (RES > 0 ? 1 : 0);  // stages
    constexpr bool NEED_B = NJ >= 1 && M >= 2; // a later stage reads sweep 1's output, u_prev where unrelaxed
    extern __shared__ unsigned char wave_smem[];
    // full (copy landed) and empty (every consumer warp done) barriers of the rings
    __shared__ unsigned long long bar_uf[kWaveMaxRing], bar_ue[kWaveMaxRing];
    __shared__ int s_fail;  // a consumer's wait ran out: the producer stops issuing copies
    __shared__ unsigned long long bar_ff[kWaveMaxRing + 2], bar_fe[kWaveMaxRing + 2];
    const WaveTile& tl = a.t;
    const int RU = tl.ru, RF = M + tl.fa;  // f ring: planes t-(M-1) .. t in use, fa in flight
    const Geom& G = a.G;
    const int P = tl.P, rows = tl.rows;
    const unsigned PB = (unsigned)P * ES;
    const unsigned SU = (unsigned)tl.slot_u, SF = (unsigned)tl.slot_f, SW = (unsigned)tl.slot_w;
    const unsigned AU = (smem_u32(wave_smem) + 127u) & ~127u;  // u0 ring
    const unsigned AF = AU + RU * SU;                           // f ring
    const unsigned AW = AF + RF * SF;                           // work planes
    const int nc = rows * tl.nvec;                              // consumer threads
    const int nwc = (nc + 31) >> 5;                             // consumer warps; the next warp is the producer
    const bool producer = (int)threadIdx.x >= nwc * 32;
    const bool lane0 = (threadIdx.x & 31u) == 0u;
    const int tile = blockIdx.x % tl.tiles_j, chunk = blockIdx.x / tl.tiles_j;
    const int j0 = tile * tl.TJ;
    const int ia = chunk * tl.ci, ib = min(G.nx, ia + tl.ci);
    // stage s computes planes [max(0, ia-(M-s)), min(nx, ib+(M-s))); u0 planes one further out
    const int lo1 = max(0, ia - (M - 1)), hi1 = min(G.nx, ib + (M - 1));
    const int lo2 = max(0, ia - (M - 2)), hi2 = min(G.nx, ib + (M - 2));
    const int pu0 = max(0, lo1 - 1), pu1 = min(G.nx, hi1 + 1);
    // consumer threads: first the interior k-vectors (1 .. nvec-2) of every row, row by row, then
    // the two end vectors (k = 0 and the one holding k = nz-1) of every row, so that the warps of
    // the interior vectors run the condition-free stencil and the few end vectors share warps
    const int nint = tl.nvec - 2;
    int r = rows, kv = 0;  // padding threads of the last consumer warp: no row
    if ((int)threadIdx.x < rows * nint) {
        r = threadIdx.x / nint;
        kv = 1 + (int)threadIdx.x - r * nint;
    } else if ((int)threadIdx.x < nc) {
        const int b = (int)threadIdx.x - rows * nint;
        r = b >> 1;
        kv = (b & 1) ? tl.nvec - 1 : 0;
    }
    const bool live = r < rows;
    const int j = j0 - (M - 1) + r, kb = kv * V;
    const bool jok = live && j >= 0 && j < G.ny;
    // all points of this vector relaxed and off the face lines (on an interior plane)
    const bool fast_col = live && kv >= 1 && kv <= tl.nvec - 2 && j >= 1 && j <= G.ny - 2;
    const int qf0 = max(1, G.x0), qf1 = min(G.nx - 1, G.x1);  // interior relaxed planes [qf0, qf1)
    const bool own_row = jok && r >= M - 1 && r < M - 1 + tl.TJ;
    unsigned ins = 0u, rjk = 0u;  // elements inside the shape / relaxed in (j, k)
    if (jok) {
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int k = kb + e;
            if (k < G.nz) {
                ins |= 1u << e;
                if (j >= G.y0 && j < G.y1 && k >= G.z0 && k < G.z1) rjk |= 1u << e;
            }
        }
    }
    const long long gjk = jok ? (long long)j * G.sy + kb : 0;  // offset of (j, kb) in a plane
    T* const Bj = a.B + gjk;
    T* const Cj = a.C + gjk;
    T* const Rj = a.r + gjk;
    const unsigned ou = (unsigned)((min(r, rows - 1) + 1) * P + kb) * ES;  // this vector in a u0 slot
    const unsigned ow = (unsigned)(min(r, rows - 1) * P + kb) * ES;        // in an f slot and in a work plane
    const int y_u = j0 - M, y_f = j0 - (M - 1);
    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int s = 0; s < RU; s++) {
            mbar_init(&bar_uf[s], 1);
            mbar_init(&bar_ue[s], nwc);
        }
        for (int s = 0; s < RF; s++) {
            mbar_init(&bar_ff[s], 1);
            mbar_init(&bar_fe[s], nwc);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // launched as a programmatic dependent: wait for the previous grid, whose writes the copies
    // (async proxy) must see
    pdl_begin();
    asm volatile("fence.proxy.async;\n" ::: "memory");
    __syncthreads();
    unsigned long long mx = 0ull;
    if (producer) {
        // ---- producer: one lane issues every copy, in the order the consumers need them (u0
        // plane p at step p-1, f plane p at step p), each into a slot its consumers released
        if (lane0) {
            // u_prev's boundary lines this tile needs: the Dirichlet k = 0 / nz-1 columns of its
            // rows and the Dirichlet j = 0 / ny-1 rows if they are among its rows
            const bool b_klo = NEED_B && G.z0 > 0, b_khi = NEED_B && G.z1 < G.nz;
            const bool b_jlo = NEED_B && G.y0 > 0 && y_f <= 0;
            const bool b_jhi = NEED_B && G.y1 < G.ny && y_f <= G.ny - 1 && G.ny - 1 < y_f + rows;
            const unsigned bytes_u = (unsigned)((rows + 2) * P) * ES + (b_klo ? (unsigned)(rows * V) * ES : 0u) +
                                     (b_khi ? (unsigned)(rows * V) * ES : 0u) + (b_jlo ? PB : 0u) + (b_jhi ? PB : 0u);
            const unsigned bytes_f = (unsigned)(rows * P) * ES;
            const int ry0 = max(0, y_u), ry1 = min(G.ny, y_u + rows + 2);  // u0 rows (L2 prefetch)
            const int fy0 = max(0, y_f), fy1 = min(G.ny, y_f + rows);      // f rows
            auto prefetch_u = [&](int p) {
                if (p >= pu1) return;
                if (tl.l2mode == 1) tma_prefetch_l2_3d(&map_u, 0, y_u, p);
                else if (tl.l2mode == 2)
                    bulk_prefetch_l2(a.A + (long long)p * G.sx + (long long)ry0 * G.sy, (unsigned)((ry1 - ry0) * G.sy) * ES);
            };
            auto prefetch_f = [&](int p) {
                if (p >= hi1) return;
                if (tl.l2mode == 1) tma_prefetch_l2_3d(&map_f, 0, y_f, p);
                else if (tl.l2mode == 2)
                    bulk_prefetch_l2(a.f + (long long)p * G.sx + (long long)fy0 * G.sy, (unsigned)((fy1 - fy0) * G.sy) * ES);
            };
            for (int p = pu0; p < pu0 + tl.l2a; p++) prefetch_u(p);
            for (int p = lo1; p < lo1 + tl.l2a; p++) prefetch_f(p);
            int nu = pu0, nf = lo1;                    // next planes
            RingPos iu{0, 1u}, jf{0, 1u};              // their slots; par: parity of the release to wait for
            // a slot's release by every consumer warp; false once a consumer has failed (no copy
            // is issued after that) or after kWaitPolls polls
            auto empty_wait = [&](unsigned long long* bar, unsigned par) -> bool {
                for (unsigned n = 0; n < kWaitPolls; n++) {
                    if (mbar_try_wait(bar, par)) return true;
                    if (*(volatile int*)&s_fail) return false;
                }
                atomicExch(a.err, 1);
                return false;
            };
            bool ok = true;
            while (ok && (nu < pu1 || nf < hi1)) {
                if (nu < pu1 && (nf >= hi1 || nu - 1 <= nf)) {
                    // the slot's previous plane must have been released (none in the first round)
                    if (nu - pu0 >= RU) ok = empty_wait(&bar_ue[iu.slot], iu.par);
                    if (!ok) break;
                    const unsigned d = AU + (unsigned)iu.slot * SU;
                    unsigned long long* bar = &bar_uf[iu.slot];
                    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                    mbar_expect_tx(bar, bytes_u);
                    tma_load_3d_s(d, &map_u, 0, y_u, nu, bar);
                    if (b_klo) tma_load_3d_s(d + tl.b_klo, &map_bk, 0, y_f, nu, bar);
                    if (b_khi) tma_load_3d_s(d + tl.b_khi, &map_bk, tl.kl, y_f, nu, bar);
                    if (b_jlo) tma_load_3d_s(d + tl.b_jlo, &map_bj, 0, 0, nu, bar);
                    if (b_jhi) tma_load_3d_s(d + tl.b_jhi, &map_bj, 0, G.ny - 1, nu, bar);
                    prefetch_u(nu + tl.l2a);
                    nu++;
                    iu.next(RU);
                } else {
                    if (nf - lo1 >= RF) ok = empty_wait(&bar_fe[jf.slot], jf.par);
                    if (!ok) break;
                    unsigned long long* bar = &bar_ff[jf.slot];
                    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                    mbar_expect_tx(bar, bytes_f);
                    tma_load_3d_s(AF + (unsigned)jf.slot * SF, &map_f, 0, y_f, nf, bar);
                    prefetch_f(nf + tl.l2a);
                    nf++;
                    jf.next(RF);
                }
            }
            // before the CTA's shared memory is released, the last copies of every slot have
            // landed (every earlier copy was waited for by the consumers before its slot was
            // released and reused)
            for (int p = max(pu0, nu - RU); p < nu; p++) {
                const int n = p - pu0;
                mbar_wait(&bar_uf[n % RU], (unsigned)(n / RU) & 1u);
            }
            for (int p = max(lo1, nf - RF); p < nf; p++) {
                const int n = p - lo1;
                mbar_wait(&bar_ff[n % RF], (unsigned)(n / RF) & 1u);
            }
        }
    } else {
        // ---- consumers
        RingPos wu{0, 0u}, wf{0, 0u};  // full barriers of the next u0 / f plane to wait for
        RingPos ru{0, 0u}, rf{0, 0u};  // empty barriers of the next u0 / f plane to release
        int nwu = pu0;                 // next u0 plane to wait for
        bool ok = true;
        auto wait_u = [&]() {
            ok = ok && wave_wait(&bar_uf[wu.slot], wu.par, a.err, a.wait_polls);
            nwu++;
            wu.next(RU);
        };
        auto wait_f = [&]() {
            ok = ok && wave_wait(&bar_ff[wf.slot], wf.par, a.err, a.wait_polls);
            wf.next(RF);
        };
        // a warp is done with a plane: every lane's reads precede lane 0's arrival
        auto release = [&](unsigned long long* bar) {
            __syncwarp();
            if (lane0) mbar_arrive(bar);
        };
        // a warp stops as a whole: its lanes' waits are combined, a failure is published to the
        // producer, and a failed warp releases nothing (no slot whose copy it did not see land)
        auto settle = [&]() {
            ok = __all_sync(0xffffffffu, ok);
            if (!ok && lane0) atomicExch(&s_fail, 1);
        };
        while (ok && nwu <= lo1 && nwu < pu1) wait_u();
        settle();
        // shared addresses of u0's planes t and t+1 and of f's planes t, t-1, t-2
        const unsigned AUend = AU + RU * SU, AFend = AF + RF * SF;
        unsigned ut = AU + (unsigned)(lo1 - pu0) * SU;
        unsigned ut1 = ut + SU == AUend ? AU : ut + SU;
        unsigned ft = AF, fq1 = AF, fq2 = AF;
        auto work = [&](int w, int p) -> unsigned { return AW + (unsigned)(2 * w + (p & 1)) * SW + ow; };
        T u0m[V];  // u0(t-1), own column: the only value carried from step to step
#pragma unroll
        for (int e = 0; e < V; e++) u0m[e] = T(0);
        if (lo1 > 0 && ok) {
            sld(u0m, AU + ou);
            release(&bar_ue[ru.slot]);  // plane lo1-1 is read only here
            ru.next(RU);
        }
        // where sweep 1 leaves u_prev's value at element e (an unrelaxed point of this vector on a
        // relaxed plane): byte offset of that value among the boundary lines copied with the u0
        // plane; on a Dirichlet x plane (every point unrelaxed) it is loaded from global memory
        unsigned boff[V];
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int k = kb + e;
            if (j < G.y0) boff[e] = tl.b_jlo + (unsigned)k * ES;
            else if (j >= G.y1) boff[e] = tl.b_jhi + (unsigned)k * ES;
            else if (k < G.z0) boff[e] = tl.b_klo + (unsigned)(r * V) * ES;
            else boff[e] = tl.b_khi + (unsigned)(r * V + k - tl.kl) * ES;
        }
        const int tend = ib + M - 1;
        // one step: stage 1 at plane t, stage 2 at t-1, stage 3 at t-2.  STEADY: every stage is
        // active at its plane and the f plane t-(M-1) is released (the middle of the chunk)
        // returns false when the consumers stop (a wait ran out)
        auto step = [&](const int t, auto steady_tag) -> bool {
            constexpr bool STEADY = decltype(steady_tag)::value;
            const bool s1 = STEADY || t < hi1;  // stage 1 at plane t
            if (s1) {
                if (t + 1 < pu1) wait_u();
                wait_f();
            }
            settle();
            if (M == 1 && !ok) return false;
            const int q2 = t - 1, q3 = t - 2;  // planes of stages 2 and 3
            const bool p2 = M >= 2 && (STEADY || (q2 >= lo2 && q2 < hi2));
            const bool p3 = M == 3 && (STEADY || (q3 >= ia && q3 < ib));
            // a failed (M >= 2) warp computes nothing and releases nothing until the rendezvous
            const bool s2 = ok && p2 && r >= 1 && r < rows - 1;
            const bool s3 = ok && p3 && own_row;
            // own-column values at the plane before a stage's plane; this thread overwrites their
            // slots in this step, so they are read first
            T x1m[V], x2m[V], o1[V], o2[V], c1[V];
            if (s2) sld(x1m, work(0, t - 2));
            if (s3) sld(x2m, work(1, t - 3));
            // ---- stage 1 at plane t: sweep 1, or the residual of u0 (NJ == 0)
            if (s1 && ok && live) {
                const unsigned Uc = ut + ou;
                T xp[V], fv[V];
                sld(c1, Uc);
                sld(xp, ut1 + ou);  // u0(t+1); not used at t = nx-1, where the east ghost replaces it
                sld(fv, ft + ow);
                const bool own_t = own_row && t >= ia && t < ib;
                if (fast_col && t >= qf0 && t < qf1) {
                    wave_fast<T, V, (NJ == 0)>(o1, c1, u0m, xp, Uc, PB, fv, a);
                    if (NJ >= 1) {
                        if ((NJ == 1 || WU1) && own_t) stv(Bj + (long long)t * G.sx, o1);
                    } else if (own_t) {
                        stv(Rj + (long long)t * G.sx, o1);
                        if (RES == 2) norm_all<T, V>(mx, o1);
                    }
                } else {
                    const bool prel = t >= G.x0 && t < G.x1;
                    const unsigned act = prel ? rjk : 0u;
                    wave_point<T, V, (NJ == 0)>(o1, c1, u0m, xp, Uc, PB, fv, act, t, j, kb, a);
                    if (NJ >= 1) {
                        // sweep 1 leaves u_prev's own values at its unrelaxed points (read by stage 2)
                        if (NEED_B) {
#pragma unroll
                            for (int e = 0; e < V; e++) {
                                if (!(((ins & ~act) >> e) & 1u)) continue;
                                if (prel) sld1(o1[e], ut + boff[e]);
                                else o1[e] = ldg(Bj + (long long)t * G.sx + e);
                            }
                        }
                        if ((NJ == 1 || WU1) && own_t && act) st_masked<T, V>(Bj + (long long)t * G.sx, o1, act);
                    } else if (own_t) {  // the residual of u0
                        if (act) st_masked<T, V>(Rj + (long long)t * G.sx, o1, act);
                        if (RES == 2) norm_act<T, V>(mx, o1, act);
                    }
                }
                if (M >= 2) sst(work(0, t), o1);
            }
            // ---- stage 2 at plane q2: sweep 2, or the residual of u1 (NJ == 1)
            if (s2) {
                const unsigned Wc = work(0, q2);
                T c[V], fv[V];
                sld(c, Wc);
                sld(fv, fq1 + ow);
                const bool own_q = own_row && q2 >= ia && q2 < ib;
                if (fast_col && q2 >= qf0 && q2 < qf1) {
                    wave_fast<T, V, (NJ == 1)>(o2, c, x1m, o1, Wc, PB, fv, a);
                    if (NJ == 2) {
                        if (own_q) stv(Cj + (long long)q2 * G.sx, o2);
                    } else if (own_q) {
                        stv(Rj + (long long)q2 * G.sx, o2);
                        if (RES == 2) norm_all<T, V>(mx, o2);
                    }
                } else {
                    const unsigned act = (q2 >= G.x0 && q2 < G.x1) ? rjk : 0u;
                    wave_point<T, V, (NJ == 1)>(o2, c, x1m, o1, Wc, PB, fv, act, q2, j, kb, a);
                    if (NJ == 2) {
                        // sweep 2 leaves u's own values (u0) at its unrelaxed points
#pragma unroll
                        for (int e = 0; e < V; e++)
                            if (!((act >> e) & 1u)) o2[e] = u0m[e];
                        if (own_q) st_masked<T, V>(Cj + (long long)q2 * G.sx, o2, ins);
                    } else if (own_q) {  // the residual of u1
                        if (act) st_masked<T, V>(Rj + (long long)q2 * G.sx, o2, act);
                        if (RES == 2) norm_act<T, V>(mx, o2, act);
                    }
                }
                if (M == 3) sst(work(1, q2), o2);
            }
            // ---- stage 3 at plane q3: the residual of u2
            if (s3) {
                const unsigned Wc = work(1, q3);
                T c[V], fv[V], out[V];
                sld(c, Wc);
                sld(fv, fq2 + ow);
                if (fast_col && q3 >= qf0 && q3 < qf1) {
                    wave_fast<T, V, true>(out, c, x2m, o2, Wc, PB, fv, a);
                    stv(Rj + (long long)q3 * G.sx, out);
                    if (RES == 2) norm_all<T, V>(mx, out);
                } else {
                    const unsigned act = (q3 >= G.x0 && q3 < G.x1) ? rjk : 0u;
                    wave_point<T, V, true>(out, c, x2m, o2, Wc, PB, fv, act, q3, j, kb, a);
                    if (act) st_masked<T, V>(Rj + (long long)q3 * G.sx, out, act);
                    if (RES == 2) norm_act<T, V>(mx, out, act);
                }
            }
            // u0 plane t and f plane t-(M-1) are no longer read
            if (s1 && ok) {
#pragma unroll
                for (int e = 0; e < V; e++) u0m[e] = c1[e];
                release(&bar_ue[ru.slot]);
                ru.next(RU);
            }
            if (ok && (STEADY || (t - (M - 1) >= lo1 && t - (M - 1) < hi1))) {
                release(&bar_fe[rf.slot]);
                rf.next(RF);
            }
            // the consumers' rendezvous of the step: this step's work-plane writes are read, and
            // this step's work-plane reads are overwritten, only after it; it also tells every
            // consumer whether one of them failed
            if (M >= 2) {
                unsigned any_fail;
                asm volatile(
                    "{\n .reg .pred pf, pa;\n setp.eq.u32 pf, %1, 0;\n bar.red.or.pred pa, 1, %2, pf;\n"
                    " selp.u32 %0, 1, 0, pa;\n}\n"
                    : "=r"(any_fail)
                    : "r"(ok ? 1u : 0u), "r"(nwc * 32)
                    : "memory");
                if (any_fail) return false;
            }
            // ring positions move one plane on
            ut = ut1;
            ut1 = ut1 + SU == AUend ? AU : ut1 + SU;
            fq2 = fq1;
            fq1 = ft;
            ft = ft + SF == AFend ? AF : ft + SF;
            return true;
        };
        // every consumer takes every step (the step's barrier counts them all); after a wait
        // ran out (error flag set) the results are invalid and the remaining waits are skipped
        int A = lo1 + M - 1, B = hi1;  // the steady steps [A, B)
        if (M >= 2) {
            A = max(A, lo2 + 1);
            B = min(B, hi2 + 1);
        }
        if (M == 3) {
            A = max(A, ia + 2);
            B = min(B, ib + 2);
        }
        B = max(A, B);
        int t = lo1;
        bool go = true;
        for (; go && t < min(A, tend); t++) go = step(t, std::false_type{});
        for (; go && t < B; t++) go = step(t, std::true_type{});
        for (; go && t < tend; t++) go = step(t, std::false_type{});
        if (RES == 2 && ok && own_row) {
            // the stored r at the tile's unrelaxed points counts in the norm too; read after the
            // march, where the loads of all planes overlap
#pragma unroll 4
            for (int q = ia; q < ib; q++) {
                const unsigned m = ins & ~((q >= G.x0 && q < G.x1) ? rjk : 0u);
                if (m) {
                    const T* rp = Rj + (long long)q * G.sx;
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if ((m >> e) & 1u) mx = max(mx, abs_bits(ldg(rp + e)));
                }
            }
        }
    }
    // the producer lane waited for its last copies, so none lands after the CTA exits
    if (RES == 2) block_max_to(mx, a.norm);
}

}  // namespace mgp
