// mgp_sweep_pair.cuh -- two weighted-Jacobi sweeps in one pass over a large level.
//
// Relaxation<T>::relax with Jacobi (include/relaxation.h:19-94, include/jacobi.h:38-83) makes
// nsmooth sweeps, each reading u_prev and writing u after swap_u.  Two consecutive sweeps
//     u1 = J(u0),  u2 = J(u1)
// read the level twice and write it twice.  This kernel marches the level once: at plane q it
// forms u1(q) from u0(q-1..q+1) and, one plane behind, u2(q-1) from u1(q-2..q), with every
// value and every operation of the two sweeps as the reference makes them (the same
// expressions in the same order, the same Neumann ghost formula applied to u0 for the first
// sweep and to u1 for the second).
//
// Buffers.  The reference's pair leaves u = u2 in the buffer that held u0 and u_prev = u1 in the
// other; its points outside the relaxation bounds (Dirichlet faces) are never written, so each
// buffer keeps its own values there.  Writing u2 over u0 in one pass is not possible (other
// CTAs still read u0), so u2 goes to a third buffer `out`, which becomes u:
//   * out  : u2 at relaxed points, u0's own values (the u buffer's) at the other points;
//   * prev : u1 at relaxed points when WRITE_U1 (the other points are only read: sweep 2 takes
//            its values there, as the reference's second sweep reads u_prev there);
//   * src  : u0, read only; the engine keeps it as the spare buffer.
// Without WRITE_U1 the relaxed points of prev keep stale values; the engine asks for that only
// where a later sweep of the same level overwrites them before anything reads them.
//
// Data movement: a CTA owns a tile of TJ rows (j) x all k of the level and marches along i.
// Its threads cover TJ+2 rows (the tile and one row each side, whose u1 the second sweep needs
// as neighbours).  Planes of u0 (TJ+4 rows), f and, where the first sweep keeps points, u_prev
// (TJ+2 rows) are staged by per-thread 16-byte cp.async into shared-memory rings two and three
// planes ahead of use; u1 of the current and previous plane lives in a shared double buffer.
// No global load waits inside a plane step except Neumann face data.  One __syncthreads per
// plane.  The (tile, plane) pairs of the level are cut into gridDim.x equal contiguous ranges,
// one per CTA.
//
// Used only with MGP_FLAG_SWEEP_PAIRS.  Measured on B200 (513x257x129 FP64, bench workload):
// 307-330 us per pair against 2 x 85 us for two single sweeps; removing the spills (768-thread
// tiles) or every global load inside the plane step moved it by less than 10%.  The copies of
// a plane are issued after the per-plane barrier and waited for two planes later; with ~66 KB
// in flight per CTA and ~4 us per plane step the kernel is short of bytes in flight.
#pragma once

namespace mgp {

#ifndef MGP_PAIR_MAX_THREADS
#define MGP_PAIR_MAX_THREADS 1024
#endif
constexpr int kPairMaxThreads = MGP_PAIR_MAX_THREADS;  // threads per CTA (launch bound)
constexpr int kPairRingU = 4;  // u0 planes: q, q+1 in use, q+2, q+3 in flight
constexpr int kPairRingF = 3;  // f planes: q in use, q+1, q+2 in flight

template <typename T>
struct PairArgs {
    Geom G;
    const T* src;   // u0 (the level's u)
    T* prev;        // u_prev: relaxed points <- u1 (WRITE_U1); other points read
    T* out;         // <- u2 (becomes the level's u)
    const T* f;
    Faces<T> F;
    T two_h, hsq, one_omega, omega_sixth;
    int tj;         // rows per tile
    int nvec;       // vectors per row = ceil(nz / V); blockDim.x = (tj + 2) * nvec
    long long work; // tiles * nx
};

__host__ __device__ constexpr size_t pair_smem_elems(int tj, int nvec, int V) {
    // u0 ring (tj+4 rows); f and u_prev rings (tj+2 rows); u1 double buffer (tj+2 rows)
    return ((size_t)kPairRingU * (tj + 4) + 2u * kPairRingF * (tj + 2) + 2u * (tj + 2)) * (size_t)nvec * V;
}

__device__ __forceinline__ void cp_async16_l2(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// One Jacobi update of a point vector:  u = one_omega*c + omega_sixth*(sum - hsq*f)
// (jacobi.h:59-61), with sum = x- + x+ + y- + y+ + z- + z+ in the reference's order.  The z
// neighbours of the vector's end elements come in as `left` / `right`; the k = 0 and k = nz-1
// Neumann ghosts replace them where the vector holds those points (kz0: element 0 is k = 0;
// ez1: the element index of k = nz-1, or V when the vector does not hold it).
template <typename T, int V>
__device__ __forceinline__ void jacobi_vec(T (&out)[V], const T (&c)[V], const T (&xm)[V], const T (&xp)[V],
                                           const T (&ym)[V], const T (&yp)[V], T left, T right, const T (&f)[V],
                                           bool kz0, T gbot, int ez1, T gtop, T m2h, T two_h, T hsq, T c1, T c6) {
#pragma unroll
    for (int e = 0; e < V; e++) {
        const T below = e > 0 ? c[e - 1] : (kz0 ? m2h * gbot + c[1] : left);
        T above = e < V - 1 ? c[e + 1] : right;
        if (e == ez1) above = two_h * gtop + below;
        const T sum = xm[e] + xp[e] + ym[e] + yp[e] + below + above;
        out[e] = c1 * c[e] + c6 * (sum - hsq * f[e]);
    }
}

template <typename T, bool WRITE_U1>
__global__ void __launch_bounds__(kPairMaxThreads, 1) k_jacobi_pair(PairArgs<T> a) {
    constexpr int V = VecT<T>::V;
    extern __shared__ __align__(16) unsigned char pair_smem[];
    const int nvec = a.nvec, P = nvec * V, R = a.tj + 2, S = R + 2;
    const int nx = a.G.nx, ny = a.G.ny, nz = a.G.nz;
    const long long sx = a.G.sx, sy = a.G.sy;
    T* ring_u = reinterpret_cast<T*>(pair_smem);
    T* ring_f = ring_u + kPairRingU * S * P;
    T* ring_p = ring_f + kPairRingF * R * P;  // u_prev at the points the first sweep keeps
    T* buf1 = ring_p + kPairRingF * R * P;
    const int r = threadIdx.x / nvec;
    const int kb = (threadIdx.x - r * nvec) * V;
    const int ou = (r + 1) * P + kb;  // this vector in a u0 slot
    const int of = r * P + kb;        // in an f slot and in a u1 buffer
    const unsigned full = (1u << V) - 1u;
    const T two_h = a.two_h, m2h = -two_h, hsq = a.hsq, c1 = a.one_omega, c6 = a.omega_sixth;
    const bool kz0 = kb == 0;
    const int ez1 = nz - 1 - kb < V ? nz - 1 - kb : V;
    pdl_begin();
    const long long per = (a.work + gridDim.x - 1) / gridDim.x;
    long long w = (long long)blockIdx.x * per;
    const long long w_end = min(a.work, w + per);
    while (w < w_end) {
        const int tile = (int)(w / nx);
        const int ia = (int)(w - (long long)tile * nx);
        const int ib = (int)min((long long)nx, ia + (w_end - w));
        w += ib - ia;
        const int j = tile * a.tj - 1 + r;  // this thread's row
        const bool jv = j >= 0 && j < ny;
        const bool inner = jv && r >= 1 && r <= R - 2;
        // ghosts are formed only where the point they serve is relaxed (Neumann faces)
        const bool jlo = j == 0 && j >= a.G.y0, jhi = j == ny - 1 && j < a.G.y1;
        unsigned ins = 0u, rjk = 0u;  // elements inside the shape / relaxed in (j, k)
        if (jv) {
#pragma unroll
            for (int e = 0; e < V; e++) {
                const int k = kb + e;
                if (k < nz) ins |= 1u << e;
                if (k < nz && j >= a.G.y0 && j < a.G.y1 && k >= a.G.z0 && k < a.G.z1) rjk |= 1u << e;
            }
        }
        const bool zlo = kz0 && (rjk & 1u), zhi = ez1 < V && ((rjk >> ez1) & 1u);
        const long long gjk = (long long)j * sy + kb;
        const T* src_jk = a.src + gjk;
        const T* f_jk = a.f + gjk;
        const T* p_jk = a.prev + gjk;
        const int jc = jv ? j : 0;  // face rows of this thread (valid only where used)
        const bool cp_lo = r == 0 && j >= 1, cp_hi = r == R - 1 && j + 1 < ny;
        const int qa = max(ia - 1, 0);
        const int ulast = min(ib + 1, nx - 1);  // last u0 plane staged
        const int flast = min(ib, nx - 1);      // last f plane staged
        auto stage_u = [&](int pu) {
            if (pu <= ulast && jv) {
                T* slot = ring_u + (pu & (kPairRingU - 1)) * S * P;
                const T* g = src_jk + (long long)pu * sx;
                cp_async16_l2(slot + ou, g);
                if (cp_lo) cp_async16_l2(slot + kb, g - sy);
                if (cp_hi) cp_async16_l2(slot + (S - 1) * P + kb, g + sy);
            }
        };
        // f, and u_prev where the first sweep keeps it (a copy may catch relaxed elements that
        // another CTA is writing; only the kept elements are read from it)
        auto stage_f = [&](int pf, int fs) {
            if (pf <= flast && jv) {
                cp_async16_l2(ring_f + fs * R * P + of, f_jk + (long long)pf * sx);
                const unsigned actp = (pf >= a.G.x0 && pf < a.G.x1) ? rjk : 0u;
                if (actp != full) cp_async16_l2(ring_p + fs * R * P + of, p_jk + (long long)pf * sx);
            }
        };
        // prologue: {u0(qa), u0(qa+1), f(qa)}, {u0(qa+2), f(qa+1)}, {u0(qa+3), f(qa+2)}
        int fs = qa % kPairRingF;  // f slot of plane q
        stage_u(qa);
        stage_u(qa + 1);
        stage_f(qa, fs);
        cp_async_commit();
        stage_u(qa + 2);
        stage_f(qa + 1, fs == 2 ? 0 : fs + 1);
        cp_async_commit();
        stage_u(qa + 3);
        stage_f(qa + 2, fs == 0 ? 2 : fs - 1);
        cp_async_commit();
        T am[V], fp[V], bmm[V], bm[V];  // u0(q-1), f(q-1), u1(q-2), u1(q-1) of this column
        if (qa > 0 && jv) ldv(am, src_jk + (long long)(qa - 1) * sx);
        else {
#pragma unroll
            for (int e = 0; e < V; e++) am[e] = T(0);
        }
#pragma unroll
        for (int e = 0; e < V; e++) fp[e] = bmm[e] = bm[e] = T(0);
        cp_async_wait<2>();
        __syncthreads();
        for (int q = qa; q <= ib; q++) {
            const int o = q - 1;
            T ac[V], fc[V], bc[V];
            // ---- first sweep: u1(q) on the tile's rows and the two halo rows
            if (q < nx && jv) {
                const T* Uc = ring_u + (q & (kPairRingU - 1)) * S * P + ou;
                lds_v(ac, Uc);
                lds_v(fc, ring_f + fs * R * P + of);
                T ap[V], ym[V], yp[V];
                lds_v(ym, Uc - P);
                lds_v(yp, Uc + P);
                const T left = Uc[-1], right = Uc[V];  // in-bounds slot reads; unused at k = 0, nz-1
                if (q + 1 < nx) {
                    lds_v(ap, ring_u + ((q + 1) & (kPairRingU - 1)) * S * P + ou);
                } else {  // east ghost  2h*gE + u(nx-2)
#pragma unroll
                    for (int e = 0; e < V; e++) ap[e] = two_h * ldg(a.F.g[F_EAST] + (long long)jc * nz + kb + e) + am[e];
                }
                T xm[V];
#pragma unroll
                for (int e = 0; e < V; e++) xm[e] = am[e];
                if (q == 0) {  // west ghost  -2h*gW + u(1)
#pragma unroll
                    for (int e = 0; e < V; e++) xm[e] = m2h * ldg(a.F.g[F_WEST] + (long long)jc * nz + kb + e) + ap[e];
                }
                if (jlo) {  // south ghost  -2h*gS + u(j=1)
                    const T* g = a.F.g[F_SOUTH] + (long long)q * nz + kb;
#pragma unroll
                    for (int e = 0; e < V; e++) ym[e] = m2h * ldg(g + e) + yp[e];
                }
                if (jhi) {  // north ghost  2h*gN + u(j=ny-2)
                    const T* g = a.F.g[F_NORTH] + (long long)q * nz + kb;
#pragma unroll
                    for (int e = 0; e < V; e++) yp[e] = two_h * ldg(g + e) + Uc[e - P];
                }
                const T gbot = zlo ? ldg(a.F.g[F_BOTTOM] + (long long)q * ny + jc) : T(0);
                const T gtop = zhi ? ldg(a.F.g[F_TOP] + (long long)q * ny + jc) : T(0);
                jacobi_vec<T, V>(bc, ac, xm, ap, ym, yp, left, right, fc, kz0, gbot, ez1, gtop, m2h, two_h, hsq, c1, c6);
                // points the first sweep leaves alone keep u_prev's value, which the reference's
                // second sweep reads there; points outside the shape are never read
                const unsigned act = (q >= a.G.x0 && q < a.G.x1) ? rjk : 0u;
                if (act != full) {
                    T pk[V];
                    lds_v(pk, ring_p + fs * R * P + of);
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if (!((act >> e) & 1u)) bc[e] = ((ins >> e) & 1u) ? pk[e] : T(0);
                }
                T* b1 = buf1 + (q & 1) * R * P + of;
#pragma unroll
                for (int e = 0; e < V; e++) b1[e] = bc[e];
                if (WRITE_U1 && inner && act && q >= ia && q < ib) {
                    T* pp = a.prev + (long long)q * sx + gjk;
                    if (act == full) {
                        stv(pp, bc);
                    } else {
#pragma unroll
                        for (int e = 0; e < V; e++)
                            if ((act >> e) & 1u) pp[e] = bc[e];
                    }
                }
            }
            // ---- second sweep: u2(o), o = q-1, on the tile's rows
            if (inner && o >= ia) {
                const unsigned act = (o >= a.G.x0 && o < a.G.x1) ? rjk : 0u;
                T u2[V];
                if (act) {
                    const T* Bc = buf1 + (o & 1) * R * P + of;
                    T xm[V], xp[V], ym[V], yp[V];
                    lds_v(ym, Bc - P);
                    lds_v(yp, Bc + P);
                    const T left = Bc[-1], right = Bc[V];
#pragma unroll
                    for (int e = 0; e < V; e++) {
                        xm[e] = bmm[e];
                        xp[e] = bc[e];
                    }
                    if (o == 0) {  // west ghost  -2h*gW + u1(1)
#pragma unroll
                        for (int e = 0; e < V; e++) xm[e] = m2h * ldg(a.F.g[F_WEST] + (long long)jc * nz + kb + e) + bc[e];
                    }
                    if (o + 1 == nx) {  // east ghost  2h*gE + u1(nx-2)
#pragma unroll
                        for (int e = 0; e < V; e++) xp[e] = two_h * ldg(a.F.g[F_EAST] + (long long)jc * nz + kb + e) + bmm[e];
                    }
                    if (jlo) {
                        const T* g = a.F.g[F_SOUTH] + (long long)o * nz + kb;
#pragma unroll
                        for (int e = 0; e < V; e++) ym[e] = m2h * ldg(g + e) + yp[e];
                    }
                    if (jhi) {
                        const T* g = a.F.g[F_NORTH] + (long long)o * nz + kb;
#pragma unroll
                        for (int e = 0; e < V; e++) yp[e] = two_h * ldg(g + e) + Bc[e - P];
                    }
                    const T gbot = zlo ? ldg(a.F.g[F_BOTTOM] + (long long)o * ny + j) : T(0);
                    const T gtop = zhi ? ldg(a.F.g[F_TOP] + (long long)o * ny + j) : T(0);
                    jacobi_vec<T, V>(u2, bm, xm, xp, ym, yp, left, right, fp, kz0, gbot, ez1, gtop, m2h, two_h, hsq, c1, c6);
                }
                // out takes u2 at relaxed points and the u buffer's own values elsewhere
#pragma unroll
                for (int e = 0; e < V; e++)
                    if (!((act >> e) & 1u)) u2[e] = am[e];
                T* po = a.out + (long long)o * sx + gjk;
                if (ins == full) {
                    stv(po, u2);
                } else {
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if ((ins >> e) & 1u) po[e] = u2[e];
                }
            }
            // ---- the column registers move one plane on
            if (q < nx && jv) {
#pragma unroll
                for (int e = 0; e < V; e++) {
                    am[e] = ac[e];
                    fp[e] = fc[e];
                    bmm[e] = bm[e];
                    bm[e] = bc[e];
                }
            }
            // u0(q+2) and f(q+1) have landed (one later group may still be in flight); after
            // the barrier the slots of u0(q) and f(q) take u0(q+4) and f(q+3)
            cp_async_wait<1>();
            __syncthreads();
            stage_u(q + 4);
            stage_f(q + 3, fs);
            cp_async_commit();
            fs = fs == kPairRingF - 1 ? 0 : fs + 1;
        }
        cp_async_wait<0>();
        __syncthreads();  // the next segment's copies reuse the rings
    }
}

}  // namespace mgp
