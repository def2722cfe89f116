// mgp_tail.cuh -- the coarsest levels of a cycle in one CTA (included by mgp_engine.cu).
//
// From level T down (T >= 1, chosen so that every field of levels T..L-1 fits in one CTA's
// shared memory: levels 4-5 of 513x257x129, about 207 KB in FP64), one V(T) or F(T) visit of
// the cycle (include/vcycle.h:14-98, include/fcycle.h:13-97) runs as ONE launch of one block:
// the block copies u (both Jacobi buffers), f, r and the face data of those levels from global
// memory into shared memory, performs the visit's operations with a block barrier between
// them, and writes everything back.  The levels' kernels and their per-launch cost (3-5 us
// each, 35 launches per F-cycle iteration on that workload) become one launch per visit.
// Measured slower on B200 (see tail_level in mgp_engine.cu), so it runs only on request
// (MGP_TUNE_TAIL), e.g. when the autotuner finds it faster.
//
// Each operation writes what the grid kernels write, with their arithmetic:
//   sweep      relaxed points of the destination (Jacobi: the other buffer; red-black: the
//              active colour in place), Neumann ghosts (sign*2h)*g + mirror, jacobi.h:59-61
//   set-up     residual at the relaxed points (residual.h) into the shared-memory r only (the
//              grid path's one-kernel set-up leaves r unstored there too), restriction into
//              f_{l+1} at every coarse point (fw_sum / injection), u_{l+1} = 0 everywhere,
//              Neumann face restriction (neumann.h:146-252)
//   prolong    u += P e at every shape point, r = P e at the unrelaxed points (the fused form)
// The coarse first sweep is computed as an ordinary sweep of the zeroed u (the grid path fuses
// it into the set-up; same expression, same values).
#pragma once

namespace mgp {

constexpr int kTailMaxLevels = 4;
constexpr int kTailThreads = 1024;

template <typename T>
struct TailLevel {
    Geom G;            // grid geometry (global strides, relaxation bounds, colour offset)
    T* ub[2];          // global u buffers (ub[1] null for Gauss-Seidel)
    T* f;
    T* r;
    T* g[6];           // global face arrays
    int gn[6];         // face elements
    int neumann[6];
    T two_h, hsq, inv_hsq, one_omega, omega_sixth, h;
    int pow2;
    int so_u[2], so_f, so_r, so_g[6];  // shared-memory offsets (elements)
};

// The visit as a flat program of level operations, written by the host from the recursion of
// vcycle_t / fcycle_t (the kernel has no recursion: its stack would not be sized statically).
enum TailOp : unsigned char { TAIL_RELAX = 0, TAIL_RELAX_SKIP1 = 1, TAIL_SETUP = 2, TAIL_PROLONG = 3 };
constexpr int kTailMaxOps = 96;

template <typename T>
struct TailArgs {
    TailLevel<T> L[kTailMaxLevels];
    int nl;          // levels in the tail
    int ns;
    int jacobi;
    int fw;          // FullWeighting (else Injection)
    int cur[kTailMaxLevels];
    int alt;         // GaussSeidel::alternate
    int nops;
    unsigned char op[kTailMaxOps], lv[kTailMaxOps];
};

template <typename T>
struct TailState {
    int cur[kTailMaxLevels];
    int alt;
};

template <typename T>
__device__ __forceinline__ int tail_idx(const Geom& G, int i, int j, int k) {
    return (i * G.ny + j) * G.nz + k;
}

// One Jacobi sweep (src -> dst) or red-black half-sweep (in place, colour) of level L.
template <typename T>
__device__ void tail_sweep(const TailLevel<T>& L, T* sm, const T* src, T* dst, int gs, int colour) {
    const Geom& G = L.G;
    const T* f = sm + L.so_f;
    const int n = G.nx * G.ny * G.nz;
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        const int k = p % G.nz, q = p / G.nz;
        const int j = q % G.ny, i = q / G.ny;
        if (i < G.x0 || i >= G.x1 || j < G.y0 || j >= G.y1 || k < G.z0 || k >= G.z1) continue;
        if (gs && ((i + j + k + G.poff) & 1) != colour) continue;
        const T two_h = L.two_h, m2h = -L.two_h;
        const T vm = i > 0 ? src[p - G.ny * G.nz] : m2h * sm[L.so_g[F_WEST] + j * G.nz + k] + src[p + G.ny * G.nz];
        const T vp = i < G.nx - 1 ? src[p + G.ny * G.nz]
                                  : two_h * sm[L.so_g[F_EAST] + j * G.nz + k] + src[p - G.ny * G.nz];
        const T ym = j > 0 ? src[p - G.nz] : m2h * sm[L.so_g[F_SOUTH] + i * G.nz + k] + src[p + G.nz];
        const T yp = j < G.ny - 1 ? src[p + G.nz] : two_h * sm[L.so_g[F_NORTH] + i * G.nz + k] + src[p - G.nz];
        const T zm = k > 0 ? src[p - 1] : m2h * sm[L.so_g[F_BOTTOM] + i * G.ny + j] + src[p + 1];
        const T zp = k < G.nz - 1 ? src[p + 1] : two_h * sm[L.so_g[F_TOP] + i * G.ny + j] + src[p - 1];
        const T sum = vm + vp + ym + yp + zm + zp;
        dst[p] = L.one_omega * src[p] + L.omega_sixth * (sum - L.hsq * f[p]);
    }
    __syncthreads();
}

template <typename T>
__device__ void tail_relax(const TailArgs<T>& a, int l, T* sm, TailState<T>& st, bool skip_first) {
    const TailLevel<T>& L = a.L[l];
    if (a.jacobi) {
        for (int it = 0; it < a.ns; it++) {
            st.cur[l] ^= 1;  // swap_u
            if (it == 0 && skip_first) continue;
            tail_sweep(L, sm, sm + L.so_u[st.cur[l] ^ 1], sm + L.so_u[st.cur[l]], 0, 0);
        }
    } else {
        for (int it = 0; it < 2 * a.ns; it++) {
            const int colour = st.alt ? 0 : 1;
            if (!(it == 0 && skip_first)) tail_sweep(L, sm, sm + L.so_u[0], sm + L.so_u[0], 1, colour);
            st.alt = !st.alt;
        }
    }
}

// residual of level l, restriction into f_{l+1}, u_{l+1} = 0, Neumann face restriction
template <typename T>
__device__ void tail_setup(const TailArgs<T>& a, int l, T* sm, TailState<T>& st) {
    const TailLevel<T>& F = a.L[l];
    const TailLevel<T>& C = a.L[l + 1];
    const Geom& G = F.G;
    const T* u = sm + F.so_u[st.cur[l]];
    const T* f = sm + F.so_f;
    T* r = sm + F.so_r;
    const int n = G.nx * G.ny * G.nz, pl = G.ny * G.nz;
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        const int k = p % G.nz, q = p / G.nz;
        const int j = q % G.ny, i = q / G.ny;
        if (i < G.x0 || i >= G.x1 || j < G.y0 || j >= G.y1 || k < G.z0 || k >= G.z1) continue;
        const T two_h = F.two_h, m2h = -F.two_h;
        const T vm = i > 0 ? u[p - pl] : m2h * sm[F.so_g[F_WEST] + j * G.nz + k] + u[p + pl];
        const T vp = i < G.nx - 1 ? u[p + pl] : two_h * sm[F.so_g[F_EAST] + j * G.nz + k] + u[p - pl];
        const T ym = j > 0 ? u[p - G.nz] : m2h * sm[F.so_g[F_SOUTH] + i * G.nz + k] + u[p + G.nz];
        const T yp = j < G.ny - 1 ? u[p + G.nz] : two_h * sm[F.so_g[F_NORTH] + i * G.nz + k] + u[p - G.nz];
        const T zm = k > 0 ? u[p - 1] : m2h * sm[F.so_g[F_BOTTOM] + i * G.ny + j] + u[p + 1];
        const T zp = k < G.nz - 1 ? u[p + 1] : two_h * sm[F.so_g[F_TOP] + i * G.ny + j] + u[p - 1];
        const T sum = vm + vp + ym + yp + zm + zp;
        r[p] = residual_pt(f[p], sum, u[p], F.hsq, F.inv_hsq, F.pow2);
    }
    // Neumann face restriction (reads the fine faces and the fine u, not r)
    for (int fc = 0; fc < 6; fc++) {
        if (!C.neumann[fc]) continue;
        const int nf = C.gn[fc];
        int fd[3], cd[3];  // fine / coarse face array shapes
        const int fxs[3] = {G.nx, G.ny, G.nz}, cxs[3] = {C.G.nx, C.G.ny, C.G.nz};
        for (int d = 0; d < 3; d++) {
            fd[d] = fxs[d];
            cd[d] = cxs[d];
        }
        if (fc == F_EAST || fc == F_WEST) fd[0] = cd[0] = 1;
        else if (fc == F_NORTH || fc == F_SOUTH) fd[1] = cd[1] = 1;
        else fd[2] = cd[2] = 1;
        int offx = 0, offy = 0, offz = 0, ii = 0, jj = 0, kk = 0, iii = 0, jjj = 0, kkk = 0;
        T c1 = T(-3.0 / 2.0), c2 = T(2.0), c3 = T(-0.5);
        switch (fc) {
            case F_EAST: offx = G.nx / 2; ii = -1; iii = -2; break;
            case F_WEST: ii = 1; iii = 2; break;
            case F_NORTH: offy = G.ny / 2; jj = -1; jjj = -2; break;
            case F_SOUTH: jj = 1; jjj = 2; break;
            case F_TOP: offz = G.nz / 2; kk = -1; kkk = -2; break;
            default: kk = 1; kkk = 2; break;
        }
        if (fc == F_EAST || fc == F_NORTH || fc == F_TOP) {
            c3 = T(0.5);
            c2 = T(-2.0);
            c1 = T(3.0 / 2.0);
        }
        const T* gf = sm + F.so_g[fc];
        T* gc = sm + C.so_g[fc];
        for (int t = threadIdx.x; t < nf; t += blockDim.x) {
            const int ck = t % cd[2], cq = t / cd[2];
            const int cj = cq % cd[1], ci = cq / cd[1];
            T g;
            if (a.fw) {
                const int fi2 = min(fd[0] - 1, 2 * ci), fj2 = min(fd[1] - 1, 2 * cj), fk2 = min(fd[2] - 1, 2 * ck);
                auto A = [&](int x, int y, int z) -> double { return (double)gf[(x * fd[1] + y) * fd[2] + z]; };
                g = fw_sum<T>(A, max(0, fi2 - 1), fi2, min(fd[0] - 1, fi2 + 1), max(0, fj2 - 1), fj2,
                              min(fd[1] - 1, fj2 + 1), max(0, fk2 - 1), fk2, min(fd[2] - 1, fk2 + 1));
            } else {
                g = gf[((2 * ci) * fd[1] + 2 * cj) * fd[2] + 2 * ck];
            }
            const int x = 2 * (ci + offx), y = 2 * (cj + offy), z = 2 * (ck + offz);
            auto U = [&](int xx, int yy, int zz) -> T { return u[(xx * G.ny + yy) * G.nz + zz]; };
            g -= (c1 * U(x, y, z) + c2 * U(x + ii, y + jj, z + kk) + c3 * U(x + iii, y + jjj, z + kkk)) / F.h;
            gc[t] = g;
        }
    }
    __syncthreads();
    // restriction r_l -> f_{l+1} and u_{l+1} = 0 over the coarse shape
    const Geom& Cg = C.G;
    const int nc = Cg.nx * Cg.ny * Cg.nz;
    T* fcoarse = sm + C.so_f;
    T* ucoarse = sm + C.so_u[st.cur[l + 1]];
    for (int p = threadIdx.x; p < nc; p += blockDim.x) {
        const int k = p % Cg.nz, q = p / Cg.nz;
        const int j = q % Cg.ny, i = q / Cg.ny;
        T v;
        if (a.fw) {
            const int ii = min(G.nx - 1, 2 * i), jj = min(G.ny - 1, 2 * j), kk = min(G.nz - 1, 2 * k);
            auto A = [&](int x, int y, int z) -> double { return (double)r[(x * G.ny + y) * G.nz + z]; };
            v = fw_sum<T>(A, max(0, ii - 1), ii, min(G.nx - 1, ii + 1), max(0, jj - 1), jj, min(G.ny - 1, jj + 1),
                          max(0, kk - 1), kk, min(G.nz - 1, kk + 1));
        } else {
            v = r[((2 * i) * G.ny + 2 * j) * G.nz + 2 * k];
        }
        fcoarse[p] = v;
        ucoarse[p] = T(0);
    }
    __syncthreads();
}

// u_l += P u_{l+1} at every shape point; r_l = P u_{l+1} at the unrelaxed points
template <typename T>
__device__ void tail_prolong(const TailArgs<T>& a, int l, T* sm, TailState<T>& st) {
    const TailLevel<T>& F = a.L[l];
    const TailLevel<T>& C = a.L[l + 1];
    const Geom& G = F.G;
    const Geom& Cg = C.G;
    const T* uc = sm + C.so_u[st.cur[l + 1]];
    T* u = sm + F.so_u[st.cur[l]];
    T* r = sm + F.so_r;
    const int n = G.nx * G.ny * G.nz;
    auto Cv = [&](int x, int y, int z) -> T {
        return (x < Cg.nx && y < Cg.ny && z < Cg.nz) ? uc[(x * Cg.ny + y) * Cg.nz + z] : T(0);
    };
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        const int k = p % G.nz, q = p / G.nz;
        const int j = q % G.ny, i = q / G.ny;
        const int ic = i >> 1, jc = j >> 1, kc = k >> 1;
        const bool ip = i & 1, jp = j & 1, kp = k & 1;
        // the x pass (odd i: midpoint of the two coarse planes), then y, then z, as prolong_tile
        T yv[2];
        for (int q2 = 0; q2 < 2; q2++) {
            T x0 = Cv(ic, jc, kc + q2), x1 = Cv(ic, jc + 1, kc + q2);
            if (ip) {
                x0 = half_sum(x0, Cv(ic + 1, jc, kc + q2));
                x1 = half_sum(x1, Cv(ic + 1, jc + 1, kc + q2));
            }
            yv[q2] = jp ? half_sum(x0, x1) : x0;
        }
        const T e = kp ? half_sum(yv[0], yv[1]) : yv[0];
        u[p] = u[p] + e;
        if (i < G.x0 || i >= G.x1 || j < G.y0 || j >= G.y1 || k < G.z0 || k >= G.z1) r[p] = e;
    }
    __syncthreads();
}

// Global (pitched) <-> shared (compact) copies of every field and face of the tail's levels.
template <typename T, bool LOAD>
__device__ void tail_copy(const TailArgs<T>& a, T* sm) {
    for (int l = 0; l < a.nl; l++) {
        const TailLevel<T>& L = a.L[l];
        const Geom& G = L.G;
        const int n = G.nx * G.ny * G.nz;
        T* gl[4] = {L.ub[0], L.ub[1], L.f, L.r};
        const int so[4] = {L.so_u[0], L.so_u[1], L.so_f, L.so_r};
        for (int b = 0; b < 4; b++) {
            if (!gl[b]) continue;
            for (int p = threadIdx.x; p < n; p += blockDim.x) {
                const int k = p % G.nz, q = p / G.nz;
                const int j = q % G.ny, i = q / G.ny;
                const long long o = (long long)i * G.sx + (long long)j * G.sy + k;
                if (LOAD) {
                    sm[so[b] + p] = gl[b][o];
                } else {
                    // r goes back at the unrelaxed points only (where the prolongation wrote it):
                    // like the grid path's one-kernel set-up, the residual stays unstored
                    if (b == 3 && i >= G.x0 && i < G.x1 && j >= G.y0 && j < G.y1 && k >= G.z0 && k < G.z1) continue;
                    gl[b][o] = sm[so[b] + p];
                }
            }
        }
        // faces: level 0's are inputs; coarser ones are written by the tail's face restriction
        for (int fc = 0; fc < 6; fc++) {
            if (!LOAD && (l == 0 || !L.neumann[fc])) continue;
            for (int t = threadIdx.x; t < L.gn[fc]; t += blockDim.x) {
                if (LOAD) sm[L.so_g[fc] + t] = L.g[fc][t];
                else L.g[fc][t] = sm[L.so_g[fc] + t];
            }
        }
    }
}

// The arguments are copied into shared memory once: device functions then read them through a
// shared-memory reference instead of each thread taking a local copy of the parameter block.
template <typename T>
__global__ void __launch_bounds__(kTailThreads, 1) k_tail(const __grid_constant__ TailArgs<T> args) {
    extern __shared__ __align__(16) unsigned char tail_smem[];
    __shared__ TailArgs<T> a;
    T* sm = reinterpret_cast<T*>(tail_smem);
    pdl_begin();
    {
        const int* src = reinterpret_cast<const int*>(&args);
        int* dst = reinterpret_cast<int*>(&a);
        for (int w = threadIdx.x; w < (int)(sizeof(TailArgs<T>) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
    }
    __syncthreads();
    tail_copy<T, true>(a, sm);
    __syncthreads();
    TailState<T> st;
    for (int l = 0; l < kTailMaxLevels; l++) st.cur[l] = a.cur[l];
    st.alt = a.alt;
    for (int q = 0; q < a.nops; q++) {
        const int l = a.lv[q];
        switch (a.op[q]) {
            case TAIL_RELAX: tail_relax(a, l, sm, st, false); break;
            case TAIL_RELAX_SKIP1: tail_relax(a, l, sm, st, true); break;
            case TAIL_SETUP: tail_setup(a, l, sm, st); break;
            default: tail_prolong(a, l, sm, st); break;
        }
    }
    tail_copy<T, false>(a, sm);
}

}  // namespace mgp
