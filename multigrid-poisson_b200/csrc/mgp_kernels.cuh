// mgp_kernels.cuh -- sm_100a stencil kernels of the multigrid engine.
//
// Device layout (one per level, shared by u, u_prev, f and r): shape points only, no ghost
// cells, k (z) unit-stride, rows padded to a 64-byte pitch:
//     off(i,j,k) = i*sx + j*sy + k,   sy = round_up(nz, 64/sizeof(T)),  sx = sy*ny.
// Neumann ghost values are never stored: each kernel forms them where it needs them, with
// the reference's arithmetic  ghost = (sign*2h)*g + u[mirror]  (include/neumann.h:63-131),
// which is exactly what the reference writes into its ghost layer before every sweep.
//
// Arithmetic follows the reference's expressions operand for operand, including its
// promotions for T=float (double literals such as 6.0 and 0.5 promote a float expression
// to double).  The library is compiled with --fmad=false, so no multiply-add is contracted
// and FP64 results match the CPU reference bit for bit.
//
// Stencil kernels use a 2.5-D march: one thread per (j,k) column of a plane, marching i
// over a chunk of planes with u(i-1), u(i), u(i+1) in registers; in-plane neighbours come
// through the read-only data path (L1).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mgp {

enum Face { F_NORTH = 0, F_SOUTH = 1, F_EAST = 2, F_WEST = 3, F_TOP = 4, F_BOTTOM = 5 };

struct Geom {
    int nx, ny, nz;
    long long sx, sy;
    int x0, x1, y0, y1, z0, z1;  // relaxation/residual bounds (is_non_eliminated, relaxation.h:78-83)
    int poff;                    // red-black colour offset
};

template <typename T>
struct Faces {
    const T* g[6];  // dense face arrays, reference face layout
};

// Programmatic dependent launch.  Every kernel of a cycle is launched with programmatic
// stream serialisation and releases its dependents as soon as it starts: the next kernel's
// CTAs are scheduled on whatever this grid leaves free (grids are dispatched in order) and
// block in pdl_begin() until this grid has completed and its writes are visible.  The launch
// latency between dependent kernels is hidden behind the running grid.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n");
}

template <typename T>
__device__ __forceinline__ T ldg(const T* p) {
    return __ldg(p);
}

// Non-negative floating values order like their bit patterns; NaN (sign cleared) sorts
// above +inf, so a NaN residual propagates into the norm.
__device__ __forceinline__ unsigned long long abs_bits(double v) {
    return (unsigned long long)__double_as_longlong(fabs(v));
}
__device__ __forceinline__ unsigned long long abs_bits(float v) {
    return (unsigned long long)__double_as_longlong(fabs((double)v));
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Block-wide max, then one atomicMax per block.
__device__ __forceinline__ void block_max_to(unsigned long long v, unsigned long long* out) {
    __shared__ unsigned long long red[32];
    v = warp_max_u64(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        unsigned long long w = lane < nw ? red[lane] : 0ull;
        w = warp_max_u64(w);
        if (lane == 0 && w) atomicMax(out, w);
    }
}

// ------------------------------------------------------------------------------------
// Stencil ops.
enum StencilOp { OP_JACOBI = 0, OP_GS = 1, OP_GS_COLUMN = 2, OP_RESIDUAL = 3 };

template <typename T>
struct StencilArgs {
    Geom G;
    const T* src;  // u (or u_prev for Jacobi)
    T* dst;        // u for Jacobi/GS, r for the residual
    const T* f;
    Faces<T> F;
    T two_h;       // 2*h of this level (T, as the reference's two_h)
    T hsq;         // h*h (T)
    T one_omega;   // 1-omega (T)
    T omega_sixth; // omega/6 (T)
    T inv_hsq;     // 1/hsq, used only when hsq is a power of two (exact)
    int hsq_pow2;
    int colour;    // GS colour (0 red: idx%2==0, 1 black)
    int ichunk;    // planes per block
    unsigned long long* norm;  // residual: max |r| over the whole shape (nullptr: none)
};

// Residual with the reference's promotions: f - (sum - 6.0*u)/hsq (include/residual.h:70-72);
// T=float evaluates in double because of the double literal 6.0.
template <typename T>
__device__ __forceinline__ T residual_pt(T fv, T sum, T uc, T hsq, T inv_hsq, int pow2);
template <>
__device__ __forceinline__ double residual_pt(double fv, double sum, double uc, double hsq, double inv_hsq, int pow2) {
    // dividing by a power of two and multiplying by its exact reciprocal round identically
    return pow2 ? fv - (sum - 6.0 * uc) * inv_hsq : fv - (sum - 6.0 * uc) / hsq;
}
template <>
__device__ __forceinline__ float residual_pt(float fv, float sum, float uc, float hsq, float inv_hsq, int pow2) {
    const double t = (double)sum - 6.0 * (double)uc;
    return (float)((double)fv - (pow2 ? t * (double)inv_hsq : t / (double)hsq));
}

// 16-byte vectors along k: 2 doubles or 4 floats per thread.  Rows are 64-byte aligned, so
// a vector starting at a multiple of V is aligned.
template <typename T>
struct VecT;
template <>
struct VecT<double> {
    static constexpr int V = 2;
    using type = double2;
};
// FP32 vector width: 4 (16-byte vectors) or, built with -DMGP_F32_VEC=2, 2 (8-byte vectors,
// as many threads per plane as FP64).  Per-element arithmetic does not depend on it.
#ifndef MGP_F32_VEC
#define MGP_F32_VEC 4
#endif
static_assert(MGP_F32_VEC == 2 || MGP_F32_VEC == 4, "MGP_F32_VEC is 2 or 4");
template <>
struct VecT<float> {
    static constexpr int V = MGP_F32_VEC;
    using type = float4;
};

__device__ __forceinline__ void ldv(double (&d)[2], const double* p) {
    const double2 x = __ldg(reinterpret_cast<const double2*>(p));
    d[0] = x.x;
    d[1] = x.y;
}
__device__ __forceinline__ void ldv(float (&d)[4], const float* p) {
    const float4 x = __ldg(reinterpret_cast<const float4*>(p));
    d[0] = x.x;
    d[1] = x.y;
    d[2] = x.z;
    d[3] = x.w;
}
__device__ __forceinline__ void ldv(float (&d)[2], const float* p) {
    const float2 x = __ldg(reinterpret_cast<const float2*>(p));
    d[0] = x.x;
    d[1] = x.y;
}
// plain (coherent) vector loads for arrays the same kernel writes
__device__ __forceinline__ void ldv_rw(double (&d)[2], const double* p) {
    const double2 x = *reinterpret_cast<const double2*>(p);
    d[0] = x.x;
    d[1] = x.y;
}
__device__ __forceinline__ void ldv_rw(float (&d)[4], const float* p) {
    const float4 x = *reinterpret_cast<const float4*>(p);
    d[0] = x.x;
    d[1] = x.y;
    d[2] = x.z;
    d[3] = x.w;
}
__device__ __forceinline__ void ldv_rw(float (&d)[2], const float* p) {
    const float2 x = *reinterpret_cast<const float2*>(p);
    d[0] = x.x;
    d[1] = x.y;
}
__device__ __forceinline__ void stv(float* p, const float (&d)[2]) {
    *reinterpret_cast<float2*>(p) = make_float2(d[0], d[1]);
}
__device__ __forceinline__ void stv(double* p, const double (&d)[2]) {
    *reinterpret_cast<double2*>(p) = make_double2(d[0], d[1]);
}
__device__ __forceinline__ void stv(float* p, const float (&d)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(d[0], d[1], d[2], d[3]);
}

// Asynchronous global->shared copies (cp.async, cached in L1 so that neighbouring threads'
// in-plane reads of the same plane still hit L1): one V-vector of T, 16 bytes (8 for 2-float
// vectors), both addresses aligned to it.
template <typename T>
__device__ __forceinline__ void cp_async_vec(void* smem, const void* gmem) {
    constexpr int B = VecT<T>::V * (int)sizeof(T);
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// cp.async of one 4- or 8-byte element (the L1-allocating form is the only one below 16 bytes)
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"((int)sizeof(T)) : "memory");
}

// Stage the V-vector at offset o: f, except at the elements in `unr`, which take r.
template <typename T, int V>
__device__ __forceinline__ void stage_f_or_r(T* slot, const T* f, const T* r, long long o, unsigned unr) {
    if (!unr) {
        cp_async_vec<T>(slot, f + o);
    } else if (unr == (1u << V) - 1u) {
        cp_async_vec<T>(slot, r + o);
    } else {
#pragma unroll
        for (int e = 0; e < V; e++) cp_async_elem(slot + e, ((unr >> e) & 1u) ? r + o + e : f + o + e);
    }
}

template <typename T>
__device__ __forceinline__ void lds_v(T (&d)[VecT<T>::V], const T* p) {
#pragma unroll
    for (int e = 0; e < VecT<T>::V; e++) d[e] = p[e];
}

#ifndef MGP_STAGES
#define MGP_STAGES 4
#endif
constexpr int kStages = MGP_STAGES;  // planes of u and f in flight per thread

// Position t of a plane's ny x nv vectors -> row j and vector kv: the interior vectors
// (kv = 1 .. nv-2) of every row first, row by row, then the two end vectors of every row.  The
// warps of interior vectors then hold no vector on a k face, so on interior rows and planes
// they all take the condition-free stencil together.
__device__ __forceinline__ void plane_vector(int t, int ny, int nv, int& j, int& kv) {
    const int ni = nv - 2;
    if (ni < 1) {
        j = t / nv;
        kv = t - j * nv;
    } else if (t < ny * ni) {
        j = t / ni;
        kv = 1 + t - j * ni;
    } else {
        const int q = t - ny * ni;
        j = q >> 1;
        kv = (q & 1) ? nv - 1 : 0;
    }
}

// The stencil at an interior vector (every neighbour a point of the level, every point
// relaxed): the relaxation or the residual of its V points from u(i-1), u(i), u(i+1), f, rows
// j-1 and j+1 and the k-1 / k+V values.  base: red-black colour of element 0.
template <typename T, int OP, bool NORM, int V>
__device__ __forceinline__ void interior_vector(const StencilArgs<T>& a, const T (&vm)[V], const T (&vc)[V],
                                                const T (&vp)[V], const T (&fc)[V], const T (&ym)[V],
                                                const T (&yp)[V], T left, T right, int base, T (&cur)[V],
                                                unsigned long long& mx) {
#pragma unroll
    for (int e = 0; e < V; e++) {
        const T below = e > 0 ? vc[e - 1] : left;
        const T above = e < V - 1 ? vc[e + 1] : right;
        const T sum = vm[e] + vp[e] + ym[e] + yp[e] + below + above;
        if (OP == OP_RESIDUAL) {
            const T r = residual_pt(fc[e], sum, vc[e], a.hsq, a.inv_hsq, a.hsq_pow2);
            cur[e] = r;
            if (NORM) mx = max(mx, abs_bits(r));
        } else {
            const T v = a.one_omega * vc[e] + a.omega_sixth * (sum - a.hsq * fc[e]);
            cur[e] = (OP == OP_GS && ((base + e) & 1) != a.colour) ? vc[e] : v;
        }
    }
}

// One thread owns a V-vector of k points of one (j) row and marches i over a chunk of
// planes with u(i-1), u(i), u(i+1) in registers.  The next kStages planes of u and f are
// staged by cp.async into the thread's own shared-memory slots, so each thread keeps
// 2*kStages*16 bytes in flight without a block barrier.  For small levels the chunk is a
// single plane (one point-vector per thread).  NORM adds the max-norm of the residual
// over the whole shape.
template <typename T, int OP, bool NORM, bool ONE = false>
__device__ __forceinline__ void stencil_tile(const StencilArgs<T>& a, const int bx, const int by) {
    constexpr int V = VecT<T>::V;
    __shared__ __align__(16) T stage_u[kStages][256 * V];
    // f; with NORM, the stored r in place of f at the vector's unrelaxed points
    __shared__ __align__(16) T stage_f[kStages][256 * V];
    const Geom& G = a.G;
    const int nv = (G.nz + V - 1) / V;
    const int t = bx * 256 + threadIdx.x;
    const int ia = by * a.ichunk;
    const int ib = min(G.nx, ia + a.ichunk);
    unsigned long long mx = 0ull;
    if (t < G.ny * nv) {
        int j, kv;
        plane_vector(t, G.ny, nv, j, kv);
        const int kb = kv * V;
        const long long bjk = (long long)j * G.sy + kb;
        const bool jin = j >= G.y0 && j < G.y1;
        // every point of the vector relaxed and off the face lines (on an interior plane): no
        // ghosts, no masks (column-ordered Gauss-Seidel keeps the general body)
        const bool fast = OP != OP_GS_COLUMN && nv >= 3 && kv >= 1 && kv <= nv - 2 && j >= 1 && j <= G.ny - 2;
        unsigned ins = 0u, inr = 0u;  // elements inside the shape / inside the relaxation bounds
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int k = kb + e;
            if (k < G.nz) ins |= 1u << e;
            if (jin && k >= G.z0 && k < G.z1) inr |= 1u << e;
        }
        const unsigned full = (1u << V) - 1u;
        const int i0 = max(ia, G.x0);
        const int i1 = inr ? min(ib, G.x1) : i0;
        // NORM: the max over the points this march computes and over the stored r outside the
        // relaxation bounds, which counts too (infinity_norm runs over the whole shape,
        // devicearray.h:221-237): the march's own vectors' unrelaxed lanes inside it, and here
        // the planes and rows it does not march.
        if (NORM) {
            if (!inr) {  // a row outside the bounds: every plane of the chunk, 4 loads in flight
                for (int i = ia; i < ib; i += 4) {
                    T v[4][V];
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        if (i + q < ib) ldv(v[q], a.dst + (long long)(i + q) * G.sx + bjk);
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        if (i + q < ib) {
#pragma unroll
                            for (int e = 0; e < V; e++)
                                if ((ins >> e) & 1u) mx = max(mx, abs_bits(v[q][e]));
                        }
                }
            } else {  // the chunk's planes outside [x0, x1): at most the first and the last
                for (int i = ia; i < min(ib, G.x0); i++) {
                    T v[V];
                    ldv(v, a.dst + (long long)i * G.sx + bjk);
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if ((ins >> e) & 1u) mx = max(mx, abs_bits(v[e]));
                }
                for (int i = max(ia, G.x1); i < ib; i++) {
                    T v[V];
                    ldv(v, a.dst + (long long)i * G.sx + bjk);
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if ((ins >> e) & 1u) mx = max(mx, abs_bits(v[e]));
                }
            }
        }
        if (i0 < i1) {
            // src may alias dst (in-place Gauss-Seidel): every value a thread reads belongs to
            // the colour this pass does not write, or to its own vector.
            const T* src = a.src;
            const T* f = a.f;
            const T two_h = a.two_h;
            const T m2h = -two_h;
            T* su = &stage_u[0][threadIdx.x * V];
            T* sf = &stage_f[0][threadIdx.x * V];
            const unsigned unr = 0u;  // elements that would stage r in place of f (none)
            const T* rr = a.dst;
            constexpr int SS = 256 * V;  // stage stride
            // stage s holds u(i0+s+1) and f(i0+s).  ONE (launched with one plane per block, on
            // small levels): nothing is staged; u(i+1) and f are loaded with the in-plane
            // neighbours, so every load of the thread is in flight at once -- one round trip to
            // memory instead of two (the staged march waits for its copies before it issues the
            // in-plane loads).
#pragma unroll
            for (int st = 0; st < kStages; st++) {
                if (ONE) break;
                const int p = i0 + st;
                if (p < i1) {
                    if (p + 1 < G.nx) cp_async_vec<T>(su + st * SS, src + (long long)(p + 1) * G.sx + bjk);
                    stage_f_or_r<T, V>(sf + st * SS, f, rr, (long long)p * G.sx + bjk, unr);
                }
                cp_async_commit();
            }
            T vm[V], vc[V], vp[V], fc[V], vmo[V];
            ldv(vc, src + (long long)i0 * G.sx + bjk);
            if (i0 > 0) {
                ldv(vm, src + (long long)(i0 - 1) * G.sx + bjk);
            } else {  // west ghost  -2h*gW + u(1)
                T v1[V];
                ldv(v1, src + G.sx + bjk);
#pragma unroll
                for (int e = 0; e < V; e++)
                    vm[e] = ((ins >> e) & 1u) ? m2h * ldg(a.F.g[F_WEST] + (long long)j * G.nz + kb + e) + v1[e] : T(0);
            }
#pragma unroll
            for (int e = 0; e < V; e++) vmo[e] = vm[e];
            for (int i = i0; i < i1; i++) {
                const long long p = (long long)i * G.sx + bjk;
                const int slot = (i - i0) % kStages;
                if (fast && i >= 1 && i + 1 < G.nx) {
                    // the condition-free body: every neighbour is a point of the level
                    if (ONE) {
                        ldv(vp, src + p + G.sx);
                        ldv(fc, f + p);
                    } else {
                        cp_async_wait<kStages - 1>();
                        lds_v(vp, su + slot * SS);
                        lds_v(fc, sf + slot * SS);
                        const int q = i + kStages;
                        if (q < i1) {
                            if (q + 1 < G.nx) cp_async_vec<T>(su + slot * SS, src + (long long)(q + 1) * G.sx + bjk);
                            cp_async_vec<T>(sf + slot * SS, f + (long long)q * G.sx + bjk);
                        }
                        cp_async_commit();
                    }
                    T ym[V], yp[V], cur[V];
                    ldv(ym, src + p - G.sy);
                    ldv(yp, src + p + G.sy);
                    const T left = ldg(src + p - 1), right = ldg(src + p + V);
                    interior_vector<T, OP, NORM, V>(a, vm, vc, vp, fc, ym, yp, left, right, i + j + kb + G.poff, cur,
                                                    mx);
                    stv(a.dst + p, cur);
#pragma unroll
                    for (int e = 0; e < V; e++) {
                        vmo[e] = vc[e];
                        vm[e] = OP == OP_GS ? cur[e] : vc[e];
                        vc[e] = vp[e];
                    }
                    continue;
                }
                if (!ONE) cp_async_wait<kStages - 1>();
                if (i + 1 < G.nx) {
                    if (ONE) ldv(vp, src + p + G.sx);
                    else lds_v(vp, su + slot * SS);
                } else {  // east ghost  2h*gE + u(nx-2), from before this sweep
#pragma unroll
                    for (int e = 0; e < V; e++)
                        vp[e] = ((ins >> e) & 1u) ? two_h * ldg(a.F.g[F_EAST] + (long long)j * G.nz + kb + e) + vmo[e]
                                                  : T(0);
                }
                if (ONE) ldv(fc, f + p);  // stage_f_or_r with no r lanes
                else lds_v(fc, sf + slot * SS);
                if (!ONE) {  // refill this slot with plane i+kStages
                    const int q = i + kStages;
                    if (q < i1) {
                        if (q + 1 < G.nx) cp_async_vec<T>(su + slot * SS, src + (long long)(q + 1) * G.sx + bjk);
                        stage_f_or_r<T, V>(sf + slot * SS, f, rr, (long long)q * G.sx + bjk, unr);
                    }
                    cp_async_commit();
                }
                unsigned act = inr;
                if (OP == OP_GS || OP == OP_GS_COLUMN) {
                    const int base = (OP == OP_GS ? i : 0) + j + kb + G.poff;
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if (((base + e) & 1) != a.colour) act &= ~(1u << e);
                }
                T cur[V];
#pragma unroll
                for (int e = 0; e < V; e++) cur[e] = vc[e];
                if (act) {
                    T ym[V], yp[V];
                    if (j > 0) {
                        ldv(ym, src + p - G.sy);
                    } else {  // south ghost  -2h*gS + u(j=1)
                        T w[V];
                        ldv(w, src + p + G.sy);
#pragma unroll
                        for (int e = 0; e < V; e++)
                            ym[e] = ((ins >> e) & 1u) ? m2h * ldg(a.F.g[F_SOUTH] + (long long)i * G.nz + kb + e) + w[e]
                                                      : T(0);
                    }
                    if (j < G.ny - 1) {
                        ldv(yp, src + p + G.sy);
                    } else {  // north ghost  2h*gN + u(j=ny-2)
                        T w[V];
                        ldv(w, src + p - G.sy);
#pragma unroll
                        for (int e = 0; e < V; e++)
                            yp[e] = ((ins >> e) & 1u) ? two_h * ldg(a.F.g[F_NORTH] + (long long)i * G.nz + kb + e) + w[e]
                                                      : T(0);
                    }
                    const T left = kb > 0 ? ldg(src + p - 1) : T(0);
                    const T right = kb + V < G.nz ? ldg(src + p + V) : T(0);
#pragma unroll
                    for (int e = 0; e < V; e++) {
                        if (!((act >> e) & 1u)) continue;
                        const int k = kb + e;
                        const T below = e > 0 ? vc[e - 1] : left;   // u(k-1)
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
                            // jacobi.h:59-61 / gaussseidel.h:43-45:
                            //   u = one_omega*v + omega_sixth*(sum - hsq*f)
                            cur[e] = a.one_omega * vc[e] + a.omega_sixth * (sum - a.hsq * fc[e]);
                        }
                    }
                    T* out = a.dst + p;
                    if (NORM && (ins & ~inr)) {  // stored r at this vector's unrelaxed points
                        T v[V];
                        ldv(v, out);
#pragma unroll
                        for (int e = 0; e < V; e++)
                            if (((ins & ~inr) >> e) & 1u) mx = max(mx, abs_bits(v[e]));
                    }
                    if (OP == OP_GS || OP == OP_GS_COLUMN) {
                        // the whole vector is this thread's; untouched entries keep their value
                        stv(out, cur);
                    } else if (act == full) {
                        stv(out, cur);
                    } else {
#pragma unroll
                        for (int e = 0; e < V; e++)
                            if ((act >> e) & 1u) out[e] = cur[e];
                    }
                }
#pragma unroll
                for (int e = 0; e < V; e++) {
                    vmo[e] = vc[e];
                    // in place (Gauss-Seidel) the register copy follows memory; Jacobi and the
                    // residual keep marching over the source iterate
                    vm[e] = (OP == OP_GS || OP == OP_GS_COLUMN) ? cur[e] : vc[e];
                    vc[e] = vp[e];
                }
            }
            cp_async_wait<0>();
        }
    }
    if (NORM) block_max_to(mx, a.norm);
}

template <typename T, int OP, bool NORM, bool ONE = false>
// (more resident blocks requested through __launch_bounds__ measured slower on B200: 5 per SM
// at 48 registers 85 us per level-0 sweep, 6 at 40 registers 132 us, against 80-82 us at 64)
__global__ void __launch_bounds__(256) k_stencil(StencilArgs<T> a) {
    pdl_begin();
    stencil_tile<T, OP, NORM, ONE>(a, blockIdx.x, blockIdx.y);
}

// The FP64 residual with its max-norm (the solve loop's): held to 64 registers, 4 blocks per SM
// (unbounded it takes 74 and 3 blocks).
template <bool ONE>
__global__ void __launch_bounds__(256, 4) k_residual_norm64(StencilArgs<double> a) {
    pdl_begin();
    stencil_tile<double, OP_RESIDUAL, true, ONE>(a, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------------------------------
// Restriction r_l -> f_{l+1} over the coarse shape, with u_{l+1} = 0 fused in
// (include/vcycle.h:43-50).  Works on any pair of (shape, strides) views, so the same code
// restricts the 2-D face arrays of Neumann::restrict_to.
struct View {
    int n[3];
    long long s0, s1;  // k unit-stride
};

// The FullWeighting sum at one coarse point from the clamped fine indices; A(x, y, z) reads
// fine point (x in {im, ii, ip}, y, z) as double.  Shared by the global-memory and the
// shared-memory restrictions, so both keep the same arithmetic.
template <typename T, typename L>
__device__ __forceinline__ T fw_sum(const L& A, int im, int ii, int ip, int jm, int jj, int jp, int km, int kk,
                                    int kp) {
    const double s_m = 1.0 * A(im, jm, km) + 2.0 * A(im, jj, km) + 1.0 * A(im, jp, km) + 2.0 * A(ii, jm, km) +
                       4.0 * A(ii, jj, km) + 2.0 * A(ii, jp, km) + 1.0 * A(ip, jm, km) + 2.0 * A(ip, jj, km) +
                       1.0 * A(ip, jp, km);
    T tmp = (T)s_m;
    const double s_0 = 2.0 * A(im, jm, kk) + 4.0 * A(im, jj, kk) + 2.0 * A(im, jp, kk) + 4.0 * A(ii, jm, kk) +
                       8.0 * A(ii, jj, kk) + 4.0 * A(ii, jp, kk) + 2.0 * A(ip, jm, kk) + 4.0 * A(ip, jj, kk) +
                       2.0 * A(ip, jp, kk);
    tmp = (T)((double)tmp + s_0);
    const double s_p = 1.0 * A(im, jm, kp) + 2.0 * A(im, jj, kp) + 1.0 * A(im, jp, kp) + 2.0 * A(ii, jm, kp) +
                       4.0 * A(ii, jj, kp) + 2.0 * A(ii, jp, kp) + 1.0 * A(ip, jm, kp) + 2.0 * A(ip, jj, kp) +
                       1.0 * A(ip, jp, kp);
    tmp = (T)((double)tmp + s_p);
    return (T)((double)tmp / 64.0);
}

template <typename T>
__device__ __forceinline__ T fw_point(const T* in, const View& vi, int i, int j, int k) {
    // FullWeighting::restrict_to (include/fullweighting.h:66-109): weights (1,2,1)^3/64 with
    // indices clamped to the array; sums in the reference's order, double accumulators.
    const int ii = min(vi.n[0] - 1, 2 * i), jj = min(vi.n[1] - 1, 2 * j), kk = min(vi.n[2] - 1, 2 * k);
    const int im = max(0, ii - 1), ip = min(vi.n[0] - 1, ii + 1);
    const int jm = max(0, jj - 1), jp = min(vi.n[1] - 1, jj + 1);
    const int km = max(0, kk - 1), kp = min(vi.n[2] - 1, kk + 1);
    auto A = [&](int x, int y, int z) -> double { return (double)ldg(in + x * vi.s0 + y * vi.s1 + z); };
    return fw_sum<T>(A, im, ii, ip, jm, jj, jp, km, kk, kp);
}

// fw_point for a thread of a warp whose lanes hold consecutive coarse points t of one coarse
// plane (t = j*n[2] + k).  Each fine row of the 3x3 neighbourhood is read as the aligned pair
// (2k, 2k+1) in one 2-element load; the value at 2k-1 is the second element of lane-1's pair
// when that lane holds (j, k-1), else (first lane of the warp, or k = 0) a scalar load or the
// clamped centre.  Same values and the same sums as fw_point.  Every lane of the warp must
// call it (lanes without a point with any point of the plane); the fine rows hold an odd
// number of points at an even pitch, so 2k+1 lies inside the row's pitch.
template <typename T>
__device__ __forceinline__ T fw_point_pairs(const T* in, const View& vi, int i, int j, int k) {
    const int ii = min(vi.n[0] - 1, 2 * i), jj = min(vi.n[1] - 1, 2 * j), kk = 2 * k;
    const int im = max(0, ii - 1), ip = min(vi.n[0] - 1, ii + 1);
    const int jm = max(0, jj - 1), jp = min(vi.n[1] - 1, jj + 1);
    const bool from_lane = (threadIdx.x & 31) != 0 && k > 0;
    const bool clamp_p = kk + 1 > vi.n[2] - 1;  // kp = kk
    const int X[3] = {im, ii, ip}, Y[3] = {jm, jj, jp};
    double vm[3][3], v0[3][3], vp[3][3];
#pragma unroll
    for (int x = 0; x < 3; x++)
#pragma unroll
        for (int y = 0; y < 3; y++) {
            const T* row = in + X[x] * vi.s0 + Y[y] * vi.s1;
            T pr[2];
            ldv(pr, row + kk);
            const T prev = __shfl_up_sync(0xffffffffu, pr[1], 1);
            v0[x][y] = (double)pr[0];
            vp[x][y] = (double)(clamp_p ? pr[0] : pr[1]);
            T m = pr[0];  // k = 0: km = kk
            if (k > 0) m = from_lane ? prev : ldg(row + kk - 1);
            vm[x][y] = (double)m;
        }
    // fw_sum over the positions (0, 1, 2) = (m, centre, p) of the neighbourhood along each axis
    auto A = [&](int x, int y, int z) -> double { return z == 0 ? vm[x][y] : (z == 1 ? v0[x][y] : vp[x][y]); };
    return fw_sum<T>(A, 0, 1, 2, 0, 1, 2, 0, 1, 2);
}

template <typename T>
struct RestrictArgs;

// The first relaxation of a coarse level right after the set-up zeroed its u
// (include/vcycle.h:43-50 then relaxation.h:19-94): every value it reads is the zero just
// written or a Neumann ghost (sign*2h)*g + 0, so it is a pointwise function of the restricted
// right-hand side and the coarse face data, and the restriction writes it directly.  The
// expression is the sweep's own, operand for operand, with the zeros in place.
template <typename T>
struct FirstSweep {
    int on;          // 0: the set-up only zeroes the coarse u
    int gs;          // red-black half-sweep in place (1) or Jacobi into `uw` (0)
    int colour;      // red-black colour of the half-sweep
    T* uw;           // Jacobi: the buffer the sweep writes (the zeroed one is the source)
    const T* gc[6];  // coarse face data, when already restricted (else formed inline)
    Geom G;          // coarse level (relaxation bounds, colour offset)
    T one_omega, omega_sixth, hsq, two_h;
};

template <typename T>
struct RestrictArgs {
    const T* in;
    View vi;
    T* out;
    View vo;
    T* zero_u;  // coarse u to zero alongside (nullptr: none)
    int fw;
    FirstSweep<T> fs;
};

// Offset of face-array indices (fi, fj, fk) in a dense face array of a level with ny x nz
// points per i-plane: west/east (1,ny,nz), south/north (nx,1,nz), bottom/top (nx,ny,1).
__device__ __forceinline__ long long face_offset(int fc, int ny, int nz, int fi, int fj, int fk) {
    if (fc == F_WEST || fc == F_EAST) return (long long)fj * nz + fk;
    if (fc == F_SOUTH || fc == F_NORTH) return (long long)fi * nz + fk;
    return (long long)fi * ny + fj;
}

// Value of the first sweep at coarse point (i,j,k) inside the relaxation bounds; g(face, fi,
// fj, fk) gives the coarse face value at face-array indices (fi, fj, fk).
template <typename T, typename G>
__device__ __forceinline__ T first_sweep_value(const FirstSweep<T>& w, T fc, int i, int j, int k, G g) {
    const Geom& C = w.G;
    const T z = T(0), two_h = w.two_h, m2h = -w.two_h;
    const T vm = i == 0 ? m2h * g(F_WEST, 0, j, k) + z : z;            // -2h*gW + u(1)
    const T vp = i == C.nx - 1 ? two_h * g(F_EAST, 0, j, k) + z : z;    // 2h*gE + u(nx-2)
    const T ym = j == 0 ? m2h * g(F_SOUTH, i, 0, k) + z : z;
    const T yp = j == C.ny - 1 ? two_h * g(F_NORTH, i, 0, k) + z : z;
    const T zm = k == 0 ? m2h * g(F_BOTTOM, i, j, 0) + z : z;
    const T zp = k == C.nz - 1 ? two_h * g(F_TOP, i, j, 0) + z : z;
    const T sum = vm + vp + ym + yp + zm + zp;
    return w.one_omega * z + w.omega_sixth * (sum - w.hsq * fc);
}

// The set-up's coarse write at offset o of coarse point (i,j,k): u = 0, and the first sweep
// where it is enabled.
template <typename T, typename G>
__device__ __forceinline__ void coarse_u_write(const FirstSweep<T>& w, T* zero_u, long long o, T fc, int i, int j,
                                               int k, G g) {
    if (!w.on) {
        zero_u[o] = T(0);
        return;
    }
    const Geom& C = w.G;
    const bool inside = i >= C.x0 && i < C.x1 && j >= C.y0 && j < C.y1 && k >= C.z0 && k < C.z1;
    if (w.gs) {
        const bool act = inside && ((i + j + k + C.poff) & 1) == w.colour;
        zero_u[o] = act ? first_sweep_value(w, fc, i, j, k, g) : T(0);
    } else {
        zero_u[o] = T(0);
        if (inside) w.uw[o] = first_sweep_value(w, fc, i, j, k, g);
    }
}

// Coarse plane `i` (the tile's y index), coarse points j*n[2]+k = bx*256 + thread of it.
// FS: the coarse u write may carry the first sweep (a.fs); a separate instantiation, as the
// branch alone slows the plain restriction (41.8 us -> 50.6 us at 513x257x129 on B200).
template <typename T, bool FS = false>
__device__ __forceinline__ void restrict_tile(const RestrictArgs<T>& a, const int bx, const int i) {
    const View vo = a.vo;
    const int n = vo.n[1] * vo.n[2];
    const int t = bx * 256 + (int)threadIdx.x;
    if (bx * 256 + (int)(threadIdx.x & ~31u) >= n) return;  // whole warps past the plane
    // lanes past the plane compute the last point (fw_point_pairs needs every lane of a warp)
    const int tc = min(t, n - 1);
    const int j = tc / vo.n[2];
    const int k = tc - j * vo.n[2];
    const T v = a.fw ? fw_point_pairs(a.in, a.vi, i, j, k)
                     : ldg(a.in + (2 * i) * a.vi.s0 + (2 * j) * a.vi.s1 + 2 * k);  // injection.h:63
    if (t >= n) return;
    const long long o = i * vo.s0 + j * vo.s1 + k;
    a.out[o] = v;
    if (FS) {
        auto g = [&](int fc, int fi, int fj, int fk) -> T {  // coarse faces restricted before this launch
            return ldg(a.fs.gc[fc] + face_offset(fc, vo.n[1], vo.n[2], fi, fj, fk));
        };
        coarse_u_write(a.fs, a.zero_u, o, v, i, j, k, g);
    } else if (a.zero_u) {
        a.zero_u[o] = T(0);
    }
}

// grid: ((n[1]*n[2] + 255)/256, n[0]) of the coarse view
template <typename T, bool FS>
__global__ void __launch_bounds__(256) k_restrict(RestrictArgs<T> a) {
    pdl_begin();
    restrict_tile<T, FS>(a, blockIdx.x, blockIdx.y);
}

// Neumann::restrict_to (include/neumann.h:146-252) for every Neumann face of the coarse
// level: g_c = R(g_f) - (c1*u0 + c2*u1 + c3*u2)/h_f.  blockIdx.y selects the face.
template <typename T>
struct BcRestrictArgs {
    const T* gf[6];
    T* gc[6];
    View vf[6], vc[6];
    int neumann[6];
    const T* u;  // fine u
    Geom Gf;     // fine level geometry (strides of u)
    T h;         // fine h
    bool fw;
};

// Neumann::restrict_to at one point (i,j,k) of face fc's coarse array (face-array indices).
template <typename T>
__device__ __forceinline__ T bc_restrict_value(const BcRestrictArgs<T>& a, int fc, int i, int j, int k) {
    const int nxf = a.Gf.nx, nyf = a.Gf.ny, nzf = a.Gf.nz;
    int offx = 0, offy = 0, offz = 0, ii = 0, jj = 0, kk = 0, iii = 0, jjj = 0, kkk = 0;
    T c1 = T(-3.0 / 2.0), c2 = T(2.0), c3 = T(-0.5);
    switch (fc) {
        case F_EAST: offx = nxf / 2; ii = -1; iii = -2; break;
        case F_WEST: ii = 1; iii = 2; break;
        case F_NORTH: offy = nyf / 2; jj = -1; jjj = -2; break;
        case F_SOUTH: jj = 1; jjj = 2; break;
        case F_TOP: offz = nzf / 2; kk = -1; kkk = -2; break;
        default: kk = 1; kkk = 2; break;
    }
    if (fc == F_EAST || fc == F_NORTH || fc == F_TOP) {
        c3 = T(0.5);
        c2 = T(-2.0);
        c1 = T(3.0 / 2.0);
    }
    T g = a.fw ? fw_point(a.gf[fc], a.vf[fc], i, j, k)
               : ldg(a.gf[fc] + (2 * i) * a.vf[fc].s0 + (2 * j) * a.vf[fc].s1 + 2 * k);
    const int x = 2 * (i + offx), y = 2 * (j + offy), z = 2 * (k + offz);
    auto U = [&](int xx, int yy, int zz) -> T { return ldg(a.u + xx * a.Gf.sx + yy * a.Gf.sy + zz); };
    g -= (c1 * U(x, y, z) + c2 * U(x + ii, y + jj, z + kk) + c3 * U(x + iii, y + jjj, z + kkk)) / a.h;
    return g;
}

// Work of one face: thread `tid` of `nthr` cooperating threads.
template <typename T>
__device__ __forceinline__ void bc_restrict_face(const BcRestrictArgs<T>& a, int fc, long long tid, long long nthr) {
    const View vo = a.vc[fc];
    const long long n = (long long)vo.n[0] * vo.n[1] * vo.n[2];
    for (long long t = tid; t < n; t += nthr) {
        const int k = (int)(t % vo.n[2]);
        const long long q = t / vo.n[2];
        const int j = (int)(q % vo.n[1]);
        const int i = (int)(q / vo.n[1]);
        a.gc[fc][i * vo.s0 + j * vo.s1 + k] = bc_restrict_value<T>(a, fc, i, j, k);
    }
}

template <typename T>
__device__ __forceinline__ void bc_restrict_tile(const BcRestrictArgs<T>& a, const int bx, const int fc, const int gx) {
    if (!a.neumann[fc]) return;
    bc_restrict_face(a, fc, bx * 256ll + threadIdx.x, gx * 256ll);
}

template <typename T>
__global__ void __launch_bounds__(256) k_restrict_bc(BcRestrictArgs<T> a) {
    pdl_begin();
    bc_restrict_tile(a, blockIdx.x, blockIdx.y, gridDim.x);
}

// ------------------------------------------------------------------------------------
// Coarse-grid set-up in one pass (include/vcycle.h:34-76): the residual of level l is
// formed plane by plane and never stored, restricted into f_{l+1} (Injection or
// FullWeighting), and u_{l+1} is zeroed.  Blocks past `main_blocks` restrict the Neumann
// face data instead.
//
// FullWeighting's coarse value is (((T)s_m + s_0) + s_p) / 64, each s a left-to-right sum
// over the fine planes im, ii, ip in that order (include/fullweighting.h:82-114).  A march
// in increasing i meets those planes in the same order, so every coarse point of the block
// carries its three partial sums in registers from one fine plane to the next and only one
// fine plane's residual tile lives in shared memory.  Fine plane i adds to coarse plane
// (i+1)/2 as im (odd i), i/2 as ii (even i) and (i-1)/2 as ip (odd i); the clamped first and
// last planes also act as im of plane 0 and as ip of the last plane.
//
// Block = (tkv, 2*tjc+1) threads: one thread per fine (row, k-vector) of the tile, which
// covers fine rows 2*J0-1 .. 2*(J0+tjc)-1 and fine k from 2*K0-V, so every fine point a
// coarse point of the tile reads is inside it; the first tjc*tkc threads also own one coarse
// point each.  Everything a plane needs is staged by cp.async kRingU-2 planes ahead into a
// ring of shared-memory slots: the u plane tile with one halo row and column on each side
// (each thread copies its own vector, the edge threads the halo), each thread's f vector
// (its stored r on planes outside the relaxation bounds), and, for the threads on the
// boundary rows and columns of the shape, the stored r of their unrelaxed points and the
// Neumann face values of their ghosts.  One barrier per plane: after it, the plane's data
// have landed, the slot of the plane before it is free for the next copy, and the previous
// plane's residual tile is complete for the coarse points to read.
template <typename T>
struct RRArgs {
    Geom Gf, Gc;
    const T* u;
    const T* f;
    const T* r;
    T* fc;
    T* uc;
    Faces<T> F;
    T two_h, hsq, inv_hsq;
    int hsq_pow2;
    int fw;
    int tjc, tkc, ci;
    int tiles_j, tiles_k, main_blocks, bc_blocks_per_face;
    BcRestrictArgs<T> bc;
    FirstSweep<T> fs;
};

// The set-up's write of coarse u at (I, J, K): zero, or the first sweep, whose Neumann ghosts
// take the coarse face values formed here (the face-restriction blocks of the same launch
// write the same values to the face arrays).
template <typename T>
__device__ __forceinline__ void rr_coarse_u(const RRArgs<T>& a, long long oo, T fc, int I, int J, int K) {
    auto g = [&](int face, int fi, int fj, int fk) -> T { return bc_restrict_value<T>(a.bc, face, fi, fj, fk); };
    coarse_u_write(a.fs, a.uc, oo, fc, I, J, K, g);
}

// The share of fine plane q (residual tile P, rows pre-multiplied by the tile row width) in
// the coarse point's restriction: Injection at the coarse plane q/2, or FullWeighting's
// running sums, i-major with weights (1,2,1 | 2,4,2 | 1,2,1), doubled on the ii plane.
template <typename T>
__device__ __forceinline__ void rr_accumulate(const T* P, int q, const RRArgs<T>& a, int I0, int I1, int nxf, int rm,
                                              int rj, int rp, int cm, int ck, int cp, long long o, int J, int K,
                                              double& s_m, double& s_0, double& s_p) {
    const Geom& Gc = a.Gc;
    if (!a.fw) {
        if (!(q & 1) && (q >> 1) >= I0 && (q >> 1) < I1) {  // injection.h:63
            const long long oo = (long long)(q >> 1) * Gc.sx + o;
            const T v = P[rj + ck];
            a.fc[oo] = v;
            rr_coarse_u(a, oo, v, q >> 1, J, K);
        }
        return;
    }
    auto A = [&](int row, int col) -> double { return (double)P[row + col]; };
    // w = 1 on the im and ip planes, 2 on the ii plane; `first` starts the sums
    auto add = [&](double w, bool first) {
        if (first) {
            s_m = w * A(rm, cm);
            s_0 = (2.0 * w) * A(rm, ck);
            s_p = w * A(rm, cp);
        } else {
            s_m = s_m + w * A(rm, cm);
            s_0 = s_0 + (2.0 * w) * A(rm, ck);
            s_p = s_p + w * A(rm, cp);
        }
        s_m = s_m + (2.0 * w) * A(rj, cm);
        s_m = s_m + w * A(rp, cm);
        s_0 = s_0 + (4.0 * w) * A(rj, ck);
        s_0 = s_0 + (2.0 * w) * A(rp, ck);
        s_p = s_p + (2.0 * w) * A(rj, cp);
        s_p = s_p + w * A(rp, cp);
    };
    auto finish = [&](int I) {  // (((T)s_m + s_0) + s_p) / 64
        T tmp = (T)s_m;
        tmp = (T)((double)tmp + s_0);
        tmp = (T)((double)tmp + s_p);
        const long long oo = (long long)I * Gc.sx + o;
        const T v = (T)((double)tmp / 64.0);
        a.fc[oo] = v;
        rr_coarse_u(a, oo, v, I, J, K);
    };
    if (q & 1) {
        const int Ip = (q - 1) >> 1, Im = (q + 1) >> 1;
        if (Ip >= I0 && Ip < I1) {
            add(1.0, false);
            finish(Ip);
        }
        if (Im >= I0 && Im < I1) add(1.0, true);
    } else {
        const int Ic = q >> 1;
        if (Ic >= I0 && Ic < I1) {
            if (q == 0) add(1.0, true);
            add(2.0, false);
            if (q == nxf - 1) {
                add(1.0, false);
                finish(Ic);
            }
        }
    }
}

constexpr int kRingU = 5;  // ring depth of k_resid_restrict (planes i, i+1 in use, 3 in flight)

// Shared memory of k_resid_restrict for a (tkv, rows) block: u tiles, f slots and boundary
// slots per ring stage, then two residual plane tiles.
template <typename T>
constexpr size_t rr_smem_bytes(int tkv, int rows) {
    return ((size_t)kRingU * ((rows + 2) * (tkv + 2) + tkv * rows + 2 * (2 * tkv + 2 * rows)) * VecT<T>::V +
            (size_t)2 * rows * tkv * VecT<T>::V) *
           sizeof(T);
}

// 16-byte cp.async that bypasses L1 (the block reads the data from shared memory only)
// One V-vector of T, not allocated in L1 where the size allows it (.cg exists for 16 bytes only)
template <typename T>
__device__ __forceinline__ void cp_async_vec_cg(void* smem, const void* gmem) {
    constexpr int B = VecT<T>::V * (int)sizeof(T);
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if (B == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(B) : "memory");
}

template <typename T>
__global__ void __launch_bounds__(384, 2) k_resid_restrict(RRArgs<T> a) {
    pdl_begin();
    if ((int)blockIdx.x >= a.main_blocks) {
        const int b = blockIdx.x - a.main_blocks;
        const int fc = b / a.bc_blocks_per_face;
        if (!a.bc.neumann[fc]) return;
        const long long nthr = (long long)a.bc_blocks_per_face * blockDim.x * blockDim.y;
        const long long tid = (long long)(b % a.bc_blocks_per_face) * blockDim.x * blockDim.y +
                              threadIdx.y * blockDim.x + threadIdx.x;
        bc_restrict_face(a.bc, fc, tid, nthr);
        return;
    }
    constexpr int V = VecT<T>::V;
    constexpr int SW = 2 * V;  // boundary slot: V values (stored r or S/N face), bottom and top face
    extern __shared__ __align__(16) unsigned char rr_smem[];
    const Geom& Gf = a.Gf;
    const Geom& Gc = a.Gc;
    const int TKV = blockDim.x, R = blockDim.y;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int TW = TKV * V;       // elements of one residual tile row
    const int US = TW + 2 * V;    // u tile row: V-1 pad, k halo, TW points, k halo, V-1 pad
    const int nthr = TKV * R;
    const int tid = ty * TKV + tx;
    const int NB = 2 * TKV + 2 * R;  // boundary slots per stage
    // one ring stage: u tile, f vectors, boundary slots
    const int STG = (R + 2) * US + nthr * V + NB * SW;
    T* ring = reinterpret_cast<T*>(rr_smem);
    T* rtile = ring + kRingU * STG;
    int b = blockIdx.x;
    const int tj = b % a.tiles_j;
    b /= a.tiles_j;
    const int tk = b % a.tiles_k;
    const int chunk = b / a.tiles_k;
    const int J0 = tj * a.tjc, K0 = tk * a.tkc;
    const int I0 = chunk * a.ci, I1 = min(Gc.nx, I0 + a.ci);
    const int jf0 = 2 * J0 - 1, kf0 = 2 * K0 - V;
    const int j = jf0 + ty;
    const int kb = kf0 + tx * V;
    unsigned ins = 0u, inr = 0u;
    const bool jok = j >= 0 && j < Gf.ny;
    const bool jin = j >= Gf.y0 && j < Gf.y1;
#pragma unroll
    for (int e = 0; e < V; e++) {
        const int k = kb + e;
        if (jok && k >= 0 && k < Gf.nz) {
            ins |= 1u << e;
            if (jin && k >= Gf.z0 && k < Gf.z1) inr |= 1u << e;
        }
    }
    const int ia = max(0, 2 * I0 - 1), ib = min(Gf.nx - 1, 2 * I1 - 1);  // fine planes ia..ib
    const int pend = min(ib + 1, Gf.nx - 1);                              // last u plane read
    // ---- this thread's copies, as (shared offset in a stage, global offset in a plane) ----
    const long long g_own = (long long)j * Gf.sy + kb;
    const int s_own = (ty + 1) * US + V + tx * V;
    // halo row: the first and last rows of threads also copy the row beyond them
    const int hrow = ty == 0 ? 0 : (ty == R - 1 ? R + 1 : -1);
    const int jh = jf0 - 1 + hrow;
    const bool c_hr = hrow >= 0 && jh >= 0 && jh < Gf.ny && kb >= 0 && kb < Gf.nz;
    const long long g_hr = (long long)jh * Gf.sy + kb;
    const int s_hr = hrow * US + V + tx * V;
    // halo column: the first and last threads of a row copy the point beyond them
    const int kh = tx == 0 ? kf0 - 1 : (tx == TKV - 1 ? kf0 + TW : -1);
    const bool c_hc = (tx == 0 || tx == TKV - 1) && jok && kh >= 0 && kh < Gf.nz;
    const long long g_hc = (long long)j * Gf.sy + kh;
    const int s_hc = (ty + 1) * US + (tx == 0 ? V - 1 : V + TW);
    const int s_f = (R + 2) * US + tid * V;
    // boundary slot: rows 0 / ny-1 of the shape, then the vectors holding k = 0 / nz-1
    const unsigned m_r = ins & ~inr;                                           // stored r
    const unsigned m_sn = ((j == 0 || j == Gf.ny - 1) && jin) ? inr : 0u;      // S/N ghosts
    const bool need_b = (inr & 1u) && kb == 0;                                 // bottom ghost
    int e_top = Gf.nz - 1 - kb;
    const bool need_t = e_top >= 0 && e_top < V && ((inr >> e_top) & 1u);    // top ghost
    e_top = max(0, min(V - 1, e_top));
    int bslot = -1;
    if (j == 0) bslot = tx;
    else if (j == Gf.ny - 1) bslot = TKV + tx;
    else if (kb == 0) bslot = 2 * TKV + ty;
    else if (kb <= Gf.nz - 1 && Gf.nz - 1 < kb + V) bslot = 2 * TKV + R + ty;
    const bool c_bd = bslot >= 0 && (m_r || m_sn || need_b || need_t);
    const int s_bd = (R + 2) * US + nthr * V + max(bslot, 0) * SW;
    const T* g_sn = j == 0 ? a.F.g[F_SOUTH] : a.F.g[F_NORTH];
    const T* u = a.u;
    const T* f = a.f;
    const T* r = a.r;
    // copies of plane p into ring stage `st`
    auto stage = [&](int p, int st) {
        T* S = ring + st * STG;
        if (p <= pend) {
            const long long pp = (long long)p * Gf.sx;
            if (ins) cp_async_vec_cg<T>(S + s_own, u + pp + g_own);
            if (c_hr) cp_async_vec_cg<T>(S + s_hr, u + pp + g_hr);
            if (c_hc) cp_async_elem(S + s_hc, u + pp + g_hc);
            if (p <= ib) {
                const bool inside = p >= Gf.x0 && p < Gf.x1;
                if (ins) cp_async_vec_cg<T>(S + s_f, (inside ? f : r) + pp + g_own);
                if (c_bd && inside) {
                    T* B = S + s_bd;
#pragma unroll
                    for (int e = 0; e < V; e++) {
                        if ((m_r >> e) & 1u) cp_async_elem(B + e, r + pp + g_own + e);
                        else if ((m_sn >> e) & 1u) cp_async_elem(B + e, g_sn + (long long)p * Gf.nz + kb + e);
                    }
                    if (need_b) cp_async_elem(B + V, a.F.g[F_BOTTOM] + (long long)p * Gf.ny + j);
                    if (need_t) cp_async_elem(B + V + 1, a.F.g[F_TOP] + (long long)p * Gf.ny + j);
                }
            }
        }
        cp_async_commit();
    };
    int st_fill = 0;
#pragma unroll 1
    for (int q = 0; q < kRingU - 1; q++) {
        stage(ia + q, st_fill);
        st_fill++;
    }
    const T two_h = a.two_h, m2h = -a.two_h;
    T vm[V];  // this thread's u(i-1)
    if (ins) {
        if (ia > 0) {
            ldv(vm, u + (long long)(ia - 1) * Gf.sx + g_own);
        } else {  // west ghost  -2h*gW + u(1)
            T v1[V];
            ldv(v1, u + Gf.sx + g_own);
#pragma unroll
            for (int e = 0; e < V; e++)
                vm[e] = ((ins >> e) & 1u) ? m2h * ldg(a.F.g[F_WEST] + (long long)j * Gf.nz + kb + e) + v1[e] : T(0);
        }
    }
    // this thread's coarse point (J, K) and its 3x3 fine (row, column) neighbourhood in the tile
    const int J = J0 + tid / a.tkc, K = K0 + tid % a.tkc;
    const bool owner = tid < a.tjc * a.tkc && J < Gc.ny && K < Gc.nz;
    const int rj = (2 * J - jf0) * TW, rm = (max(0, 2 * J - 1) - jf0) * TW, rp = (min(Gf.ny - 1, 2 * J + 1) - jf0) * TW;
    const int ck = 2 * K - kf0, cm = max(0, 2 * K - 1) - kf0, cp = min(Gf.nz - 1, 2 * K + 1) - kf0;
    const long long o = (long long)J * Gc.sy + K;
    double s_m = 0.0, s_0 = 0.0, s_p = 0.0;
    int st_cur = 0;  // ring stage of plane i
#pragma unroll 1
    for (int i = ia; i <= ib; i++) {
        cp_async_wait<kRingU - 3>();  // this thread's copies of planes i and i+1 have landed
        __syncthreads();
        stage(i + kRingU - 1, st_fill);  // into the stage of plane i-1, which every thread is done with
        st_fill = st_fill + 1 == kRingU ? 0 : st_fill + 1;
        const int st_nxt = st_cur + 1 == kRingU ? 0 : st_cur + 1;
        if (ins) {
            const T* S = ring + st_cur * STG;
            const T* tu = S + s_own;  // u(i) at (j, kb)
            T val[V];
            if (i >= Gf.x0 && i < Gf.x1) {
                T vc[V], vp[V], fcur[V], bd[SW];
                lds_v(vc, tu);
                if (i + 1 < Gf.nx) {
                    lds_v(vp, ring + st_nxt * STG + s_own);
                } else {  // east ghost  2h*gE + u(nx-2)
#pragma unroll
                    for (int e = 0; e < V; e++)
                        vp[e] = ((ins >> e) & 1u) ? two_h * ldg(a.F.g[F_EAST] + (long long)j * Gf.nz + kb + e) + vm[e]
                                                  : T(0);
                }
                lds_v(fcur, S + s_f);
                if (c_bd) {
#pragma unroll
                    for (int e = 0; e < SW; e++) bd[e] = S[s_bd + e];
                } else {
#pragma unroll
                    for (int e = 0; e < SW; e++) bd[e] = T(0);
                }
                T ym[V], yp[V];
                if (j > 0) {
                    lds_v(ym, tu - US);
                } else {  // south ghost  -2h*gS + u(j=1)
                    T w[V];
                    lds_v(w, tu + US);
#pragma unroll
                    for (int e = 0; e < V; e++) ym[e] = m2h * bd[e] + w[e];
                }
                if (j < Gf.ny - 1) {
                    lds_v(yp, tu + US);
                } else {  // north ghost  2h*gN + u(j=ny-2)
                    T w[V];
                    lds_v(w, tu - US);
#pragma unroll
                    for (int e = 0; e < V; e++) yp[e] = two_h * bd[e] + w[e];
                }
                const T left = kb > 0 ? tu[-1] : T(0);
                const T right = kb + V < Gf.nz ? tu[V] : T(0);
#pragma unroll
                for (int e = 0; e < V; e++) {
                    if ((m_r >> e) & 1u) {
                        val[e] = bd[e];  // stored r
                        continue;
                    }
                    if (!((inr >> e) & 1u)) {
                        val[e] = T(0);
                        continue;
                    }
                    const int k = kb + e;
                    const T below = e > 0 ? vc[e - 1] : left;
                    const T above = e < V - 1 ? vc[e + 1] : right;
                    const T zm = k > 0 ? below : m2h * bd[V] + vc[1];                     // -2h*gB + u(1)
                    const T zp = k < Gf.nz - 1 ? above : two_h * bd[V + 1] + below;       // 2h*gT + u(nz-2)
                    const T sum = vm[e] + vp[e] + ym[e] + yp[e] + zm + zp;
                    val[e] = residual_pt(fcur[e], sum, vc[e], a.hsq, a.inv_hsq, a.hsq_pow2);
                }
#pragma unroll
                for (int e = 0; e < V; e++) vm[e] = vc[e];
            } else {  // a plane outside the relaxation bounds: the stored r, staged in the f slot
                lds_v(val, S + s_f);
                T vc[V];
                lds_v(vc, tu);
#pragma unroll
                for (int e = 0; e < V; e++) vm[e] = vc[e];
            }
            stv(rtile + (i & 1) * (R * TW) + ty * TW + tx * V, val);
        }
        st_cur = st_nxt;
        if (owner && i > ia) {
            // the coarse points' share of fine plane i-1, whose residual tile is complete
            const int q = i - 1;
            const T* P = rtile + (q & 1) * (R * TW);
            rr_accumulate(P, q, a, I0, I1, Gf.nx, rm, rj, rp, cm, ck, cp, o, J, K, s_m, s_0, s_p);
        }
    }
    __syncthreads();
    if (owner)
        rr_accumulate(rtile + (ib & 1) * (R * TW), ib, a, I0, I1, Gf.nx, rm, rj, rp, cm, ck, cp, o, J, K, s_m, s_0, s_p);
    cp_async_wait<0>();
}

// ------------------------------------------------------------------------------------
// Trilinear prolongation (include/trilinearinterpolation.h:29-134), evaluated per fine
// point with the reference's pass structure: inject even points, then x, y and z midpoints
// of the previous passes' values.  ADD: u += P e (DeviceArray::add, devicearray.h:161-196);
// r receives P e on points outside the relaxation bounds (where the reference's r keeps it
// until the next prolongation) or, when !ADD, everywhere.
template <typename T>
__device__ __forceinline__ T half_sum(T a, T b) {
    return (T)(0.5 * (a + b));
}

// One thread: fine rows (2ic..2ic+1, 2jc..2jc+1) at one k-vector, from the coarse values
// (ic..ic+1, jc..jc+1, kb/2..kb/2+V/2) -- each coarse value is loaded once per thread.
template <typename T>
struct ProlongArgs {
    const T* uc;
    Geom Gc;
    T* u;
    T* r;
    Geom Gf;
};

template <typename T, bool ADD>
__device__ __forceinline__ void prolong_tile(const ProlongArgs<T>& a, const int bx, const int by) {
    constexpr int V = VecT<T>::V;
    constexpr int NQ = V / 2 + 1;
    const T* __restrict__ uc = a.uc;
    const Geom& Gc = a.Gc;
    const Geom& Gf = a.Gf;
    T* u = a.u;
    T* r = a.r;
    const int nv = (Gf.nz + V - 1) / V;
    const int t = bx * 256 + threadIdx.x;
    if (t >= Gc.ny * nv) return;
    const int ic = by;
    const int jc = t / nv;
    const int kb = (t - jc * nv) * V;  // even
    const bool i_odd_ok = 2 * ic + 1 < Gf.nx, j_odd_ok = 2 * jc + 1 < Gf.ny;
    unsigned ins = 0u;
#pragma unroll
    for (int e = 0; e < V; e++)
        if (kb + e < Gf.nz) ins |= 1u << e;
    const unsigned full = (1u << V) - 1u;
    // the four fine rows' u first: their loads do not wait for the coarse values
    T uv[2][2][V];
    bool ok[2][2];
    long long pp[2][2];
#pragma unroll
    for (int ip = 0; ip < 2; ip++)
#pragma unroll
        for (int jp = 0; jp < 2; jp++) {
            ok[ip][jp] = (!ip || i_odd_ok) && (!jp || j_odd_ok);
            pp[ip][jp] = (long long)(2 * ic + ip) * Gf.sx + (long long)(2 * jc + jp) * Gf.sy + kb;
            if (ADD && ok[ip][jp]) {
                if (ins == full) {
                    ldv_rw(uv[ip][jp], u + pp[ip][jp]);
                } else {
#pragma unroll
                    for (int e = 0; e < V; e++) uv[ip][jp][e] = ((ins >> e) & 1u) ? u[pp[ip][jp] + e] : T(0);
                }
            }
        }
    // coarse values c[a][b][q] = C(ic+a, jc+b, kb/2+q)
    T c[2][2][NQ];
#pragma unroll
    for (int a2 = 0; a2 < 2; a2++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const int x = ic + a2, y = jc + b, z = (kb >> 1) + q;
                c[a2][b][q] = (x < Gc.nx && y < Gc.ny && z < Gc.nz) ? ldg(uc + x * Gc.sx + y * Gc.sy + z) : T(0);
            }
    // the four fine rows' prolongated values
    T ev[2][2][V];
    unsigned insd[2][2];
#pragma unroll
    for (int ip = 0; ip < 2; ip++)
#pragma unroll
        for (int jp = 0; jp < 2; jp++) {
            const int i = 2 * ic + ip, j = 2 * jc + jp;
            // x pass (odd i: midpoint of the two coarse planes), then y pass, per coarse z
            T yv[NQ];
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                T x0 = c[0][0][q], x1 = c[0][1][q];
                if (ip) {
                    x0 = half_sum(x0, c[1][0][q]);
                    x1 = half_sum(x1, c[1][1][q]);
                }
                yv[q] = jp ? half_sum(x0, x1) : x0;
            }
#pragma unroll
            for (int e = 0; e < V; e++)
                ev[ip][jp][e] = (e & 1) ? half_sum(yv[e >> 1], yv[(e >> 1) + 1]) : yv[e >> 1];
            const bool ijin = i >= Gf.x0 && i < Gf.x1 && j >= Gf.y0 && j < Gf.y1;
            unsigned inside = 0u;
#pragma unroll
            for (int e = 0; e < V; e++)
                if (ijin && kb + e >= Gf.z0 && kb + e < Gf.z1) inside |= 1u << e;
            insd[ip][jp] = inside;
        }
#pragma unroll
    for (int ip = 0; ip < 2; ip++)
#pragma unroll
        for (int jp = 0; jp < 2; jp++) {
            if (!ok[ip][jp]) continue;
            const long long p = pp[ip][jp];
            if (ADD) {
                T nv[V];
#pragma unroll
                for (int e = 0; e < V; e++) nv[e] = uv[ip][jp][e] + ev[ip][jp][e];
                if (ins == full) {
                    stv(u + p, nv);
                } else {
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if ((ins >> e) & 1u) u[p + e] = nv[e];
                }
                const unsigned rm = ins & ~insd[ip][jp];
#pragma unroll
                for (int e = 0; e < V; e++)
                    if ((rm >> e) & 1u) r[p + e] = ev[ip][jp][e];
            } else {
                if (ins == full) {
                    stv(r + p, ev[ip][jp]);
                } else {
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if ((ins >> e) & 1u) r[p + e] = ev[ip][jp][e];
                }
            }
        }
}

// ---- prolongation + add fused with the first Jacobi sweep after it (levels >= 1, nsmooth even) --
// u' = u + P u_c, then one sweep of u' into the other buffer, in one pass: every thread forms
// u' at its point and at the six neighbours from u and the coarse values (the arithmetic of
// prolong_tile) and sweeps (jacobi.h:59-61), writing the other buffer at relaxed points.  u' is
// not stored at relaxed points: the second sweep of the relaxation overwrites them before
// anything reads them.  At unrelaxed (Dirichlet) points P u_c is exactly +0 -- with nsmooth
// even the coarse u read here is the buffer the set-up zeroed, whose Dirichlet points stay +0
// (prolong_sweep_fused in mgp_engine.cu) -- so u there becomes u + 0 in place (a reader that
// sees the old or the new value forms the same u + 0) and r takes P u_c, as prolong_tile
// leaves it.
template <typename T>
struct ProlongSweepArgs {
    const T* uc;
    Geom Gc;
    T* u;        // current u (read; written at unrelaxed points)
    T* dst;      // the other buffer: the sweep's result at relaxed points
    const T* f;
    T* r;
    Geom Gf;
    Faces<T> F;
    T two_h, hsq, one_omega, omega_sixth;
};

template <typename T>
__device__ __forceinline__ T prolong_value(const T* __restrict__ uc, const Geom& C, int i, int j, int k) {
    auto Cv = [&](int x, int y, int z) -> T {
        return (x < C.nx && y < C.ny && z < C.nz) ? ldg(uc + x * C.sx + y * C.sy + z) : T(0);
    };
    const int ic = i >> 1, jc = j >> 1, kc = k >> 1;
    T yv[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        T x0 = Cv(ic, jc, kc + q), x1 = Cv(ic, jc + 1, kc + q);
        if (i & 1) {
            x0 = half_sum(x0, Cv(ic + 1, jc, kc + q));
            x1 = half_sum(x1, Cv(ic + 1, jc + 1, kc + q));
        }
        yv[q] = (j & 1) ? half_sum(x0, x1) : x0;
    }
    return (k & 1) ? half_sum(yv[0], yv[1]) : yv[0];
}

template <typename T>
__global__ void __launch_bounds__(256) k_prolong_sweep(ProlongSweepArgs<T> a) {
    pdl_begin();
    const Geom& G = a.Gf;
    const int t = blockIdx.x * 256 + (int)threadIdx.x;
    if (t >= G.ny * G.nz) return;
    const int i = blockIdx.y, j = t / G.nz, k = t - (t / G.nz) * G.nz;
    const long long p = (long long)i * G.sx + (long long)j * G.sy + k;
    const bool relaxed = i >= G.x0 && i < G.x1 && j >= G.y0 && j < G.y1 && k >= G.z0 && k < G.z1;
    if (!relaxed) {
        const T e = prolong_value(a.uc, a.Gc, i, j, k);
        a.u[p] = a.u[p] + e;
        a.r[p] = e;
        return;
    }
    // u' at a point of the level
    auto U = [&](int x, int y, int z) -> T {
        const long long q = (long long)x * G.sx + (long long)y * G.sy + z;
        return a.u[q] + prolong_value(a.uc, a.Gc, x, y, z);
    };
    const T two_h = a.two_h, m2h = -a.two_h;
    const T uc0 = U(i, j, k);
    const T vm = i > 0 ? U(i - 1, j, k) : m2h * ldg(a.F.g[F_WEST] + (long long)j * G.nz + k) + U(1, j, k);
    const T vp = i < G.nx - 1 ? U(i + 1, j, k) : two_h * ldg(a.F.g[F_EAST] + (long long)j * G.nz + k) + U(G.nx - 2, j, k);
    const T ym = j > 0 ? U(i, j - 1, k) : m2h * ldg(a.F.g[F_SOUTH] + (long long)i * G.nz + k) + U(i, 1, k);
    const T yp = j < G.ny - 1 ? U(i, j + 1, k) : two_h * ldg(a.F.g[F_NORTH] + (long long)i * G.nz + k) + U(i, G.ny - 2, k);
    const T zm = k > 0 ? U(i, j, k - 1) : m2h * ldg(a.F.g[F_BOTTOM] + (long long)i * G.ny + j) + U(i, j, 1);
    const T zp = k < G.nz - 1 ? U(i, j, k + 1) : two_h * ldg(a.F.g[F_TOP] + (long long)i * G.ny + j) + U(i, j, G.nz - 2);
    const T sum = vm + vp + ym + yp + zm + zp;
    a.dst[p] = a.one_omega * uc0 + a.omega_sixth * (sum - a.hsq * ldg(a.f + p));
}

template <typename T, bool ADD>
__global__ void __launch_bounds__(256) k_prolong(ProlongArgs<T> a) {
    pdl_begin();
    prolong_tile<T, ADD>(a, blockIdx.x, blockIdx.y);
}

// u += r over the shape (DeviceArray::add).
template <typename T>
__global__ void __launch_bounds__(256) k_add(T* u, const T* __restrict__ r, Geom G) {
    pdl_begin();
    const long long n = (long long)G.nx * G.ny * G.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % G.nz);
        const long long q = t / G.nz;
        const int j = (int)(q % G.ny);
        const int i = (int)(q / G.ny);
        const long long p = (long long)i * G.sx + (long long)j * G.sy + k;
        u[p] = u[p] + ldg(r + p);
    }
}

// max |a| over the shape (DeviceArray::infinity_norm).  grid: ((ny*nz + 255)/256, chunks of
// planes); each thread reads one (j, k) column of its block's planes.
template <typename T>
__global__ void __launch_bounds__(256) k_norm(const T* __restrict__ a, Geom G, unsigned long long* out) {
    pdl_begin();
    const int t = blockIdx.x * 256 + (int)threadIdx.x;
    unsigned long long mx = 0ull;
    if (t < G.ny * G.nz) {
        const int j = t / G.nz;
        const int k = t - j * G.nz;
        const T* col = a + (long long)j * G.sy + k;
        for (int i = blockIdx.y; i < G.nx; i += gridDim.y) mx = max(mx, abs_bits(ldg(col + (long long)i * G.sx)));
    }
    block_max_to(mx, out);
}

// ------------------------------------------------------------------------------------
// Iterative refinement.  The outer level keeps u, f and the boundary data in FP64; a
// correction e with A e = r and homogeneous boundary data (Dirichlet 0, Neumann ghost =
// mirror) is solved on an inner hierarchy of type Ti, then u += e.
//
// k_refine_residual: r = f - A u (the reference's residual with its ghost rule) over the
// relaxation bounds; writes (Ti) r into the inner right-hand side, zeroes the inner initial
// guess, reduces max |r|, and with WRITE_R also stores r (the user-visible residual).
template <typename T, typename Ti>
struct RefineArgs {
    Geom G;                 // outer level 0
    const T* u;
    const T* f;
    T* r;
    Faces<T> F;
    T two_h, hsq, inv_hsq;
    int hsq_pow2;
    int ichunk;
    long long sxi, syi;     // inner level-0 strides
    Ti* fi;                 // inner right-hand side
    Ti* ui;                 // inner initial guess (zeroed) / correction (read by the update)
    unsigned long long* norm;
};

template <typename T, typename Ti, bool WRITE_R>
__device__ __forceinline__ void refine_residual_tile(const RefineArgs<T, Ti>& a, const int bx, const int by) {
    constexpr int V = VecT<T>::V;
    const Geom& G = a.G;
    const int nv = (G.nz + V - 1) / V;
    const int t = bx * 256 + threadIdx.x;
    const int ia = by * a.ichunk;
    const int ib = min(G.nx, ia + a.ichunk);
    unsigned long long mx = 0ull;
    if (t < G.ny * nv) {
        const int j = t / nv;
        const int kb = (t - j * nv) * V;
        const long long bjk = (long long)j * G.sy + kb;
        const long long bjki = (long long)j * a.syi + kb;
        const bool jin = j >= G.y0 && j < G.y1;
        unsigned ins = 0u, inr = 0u;
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int k = kb + e;
            if (k < G.nz) ins |= 1u << e;
            if (jin && k >= G.z0 && k < G.z1) inr |= 1u << e;
        }
        const int i0 = max(ia, G.x0);
        const int i1 = inr ? min(ib, G.x1) : i0;
        if (i0 < i1) {
            const T two_h = a.two_h, m2h = -a.two_h;
            T vm[V], vc[V], vp[V], vpp[V], fc[V], fn[V];
            ldv(vc, a.u + (long long)i0 * G.sx + bjk);
            if (i0 > 0) {
                ldv(vm, a.u + (long long)(i0 - 1) * G.sx + bjk);
            } else {
                T v1[V];
                ldv(v1, a.u + G.sx + bjk);
#pragma unroll
                for (int e = 0; e < V; e++)
                    vm[e] = ((ins >> e) & 1u) ? m2h * ldg(a.F.g[F_WEST] + (long long)j * G.nz + kb + e) + v1[e] : T(0);
            }
            if (i0 + 1 < G.nx) ldv(vp, a.u + (long long)(i0 + 1) * G.sx + bjk);
            ldv(fc, a.f + (long long)i0 * G.sx + bjk);
            for (int i = i0; i < i1; i++) {
                const long long p = (long long)i * G.sx + bjk;
                if (i + 1 < i1) {
                    if (i + 2 < G.nx) ldv(vpp, a.u + p + 2 * G.sx);
                    ldv(fn, a.f + p + G.sx);
                }
                if (i + 1 == G.nx) {
#pragma unroll
                    for (int e = 0; e < V; e++)
                        vp[e] = ((ins >> e) & 1u) ? two_h * ldg(a.F.g[F_EAST] + (long long)j * G.nz + kb + e) + vm[e]
                                                  : T(0);
                }
                T ym[V], yp[V];
                if (j > 0) {
                    ldv(ym, a.u + p - G.sy);
                } else {
                    T w[V];
                    ldv(w, a.u + p + G.sy);
#pragma unroll
                    for (int e = 0; e < V; e++)
                        ym[e] = ((ins >> e) & 1u) ? m2h * ldg(a.F.g[F_SOUTH] + (long long)i * G.nz + kb + e) + w[e] : T(0);
                }
                if (j < G.ny - 1) {
                    ldv(yp, a.u + p + G.sy);
                } else {
                    T w[V];
                    ldv(w, a.u + p - G.sy);
#pragma unroll
                    for (int e = 0; e < V; e++)
                        yp[e] = ((ins >> e) & 1u) ? two_h * ldg(a.F.g[F_NORTH] + (long long)i * G.nz + kb + e) + w[e]
                                                  : T(0);
                }
                const T left = kb > 0 ? ldg(a.u + p - 1) : T(0);
                const T right = kb + V < G.nz ? ldg(a.u + p + V) : T(0);
                T rv[V];
#pragma unroll
                for (int e = 0; e < V; e++) {
                    rv[e] = T(0);
                    if (!((inr >> e) & 1u)) continue;
                    const int k = kb + e;
                    const T below = e > 0 ? vc[e - 1] : left;
                    const T above = e < V - 1 ? vc[e + 1] : right;
                    const T zm = k > 0 ? below : m2h * ldg(a.F.g[F_BOTTOM] + (long long)i * G.ny + j) + vc[1];
                    const T zp = k < G.nz - 1 ? above : two_h * ldg(a.F.g[F_TOP] + (long long)i * G.ny + j) + below;
                    const T sum = vm[e] + vp[e] + ym[e] + yp[e] + zm + zp;
                    rv[e] = residual_pt(fc[e], sum, vc[e], a.hsq, a.inv_hsq, a.hsq_pow2);
                    mx = max(mx, abs_bits(rv[e]));
                }
                const long long q = (long long)i * a.sxi + bjki;
#pragma unroll
                for (int e = 0; e < V; e++) {
                    if (!((inr >> e) & 1u)) continue;
                    a.fi[q + e] = (Ti)rv[e];
                    a.ui[q + e] = Ti(0);
                    if (WRITE_R) a.r[p + e] = rv[e];
                }
#pragma unroll
                for (int e = 0; e < V; e++) {
                    vm[e] = vc[e];
                    vc[e] = vp[e];
                    vp[e] = vpp[e];
                    fc[e] = fn[e];
                }
            }
        }
    }
    block_max_to(mx, a.norm);
}

template <typename T, typename Ti, bool WRITE_R>
__global__ void __launch_bounds__(256) k_refine_residual(RefineArgs<T, Ti> a) {
    pdl_begin();
    refine_residual_tile<T, Ti, WRITE_R>(a, blockIdx.x, blockIdx.y);
}

// u += (T) e over the relaxation bounds (e: the inner level-0 solution).
template <typename T, typename Ti>
struct UpdateArgs {
    T* u;
    Geom G;
    const Ti* e;
    long long sxi, syi;
};

// V values of e (type Ti) at an offset that is a multiple of V (rows of the inner level are
// 64-byte aligned): one 16-byte load, or one 8-byte load for V floats next to V doubles.
__device__ __forceinline__ void ld_corr(double (&d)[2], const double* p) { ldv(d, p); }
__device__ __forceinline__ void ld_corr(double (&d)[2], const float* p) {
    const float2 x = __ldg(reinterpret_cast<const float2*>(p));
    d[0] = (double)x.x;
    d[1] = (double)x.y;
}
__device__ __forceinline__ void ld_corr(float (&d)[4], const float* p) { ldv(d, p); }
__device__ __forceinline__ void ld_corr(float (&d)[2], const float* p) { ldv(d, p); }

// Plane i (the tile's y index): one thread per k-vector of a row, u += (T) e where
// (i, j, k) is inside the relaxation bounds.
template <typename T, typename Ti>
__device__ __forceinline__ void refine_update_tile(const UpdateArgs<T, Ti>& a, const int bx, const int i) {
    constexpr int V = VecT<T>::V;
    const Geom& G = a.G;
    const int nv = (G.nz + V - 1) / V;
    const int t = bx * 256 + (int)threadIdx.x;
    if (t >= G.ny * nv || i < G.x0 || i >= G.x1) return;
    const int j = t / nv;
    const int kb = (t - j * nv) * V;
    if (j < G.y0 || j >= G.y1) return;
    unsigned act = 0u;
#pragma unroll
    for (int e = 0; e < V; e++)
        if (kb + e >= G.z0 && kb + e < G.z1) act |= 1u << e;
    if (!act) return;
    T* up = a.u + (long long)i * G.sx + (long long)j * G.sy + kb;
    T c[V], u[V];
    ld_corr(c, a.e + (long long)i * a.sxi + (long long)j * a.syi + kb);
    ldv_rw(u, up);
#pragma unroll
    for (int e = 0; e < V; e++) u[e] = u[e] + c[e];
    if (act == (1u << V) - 1u) {
        stv(up, u);
    } else {
#pragma unroll
        for (int e = 0; e < V; e++)
            if ((act >> e) & 1u) up[e] = u[e];
    }
}

// grid: ((ny * ceil(nz/V) + 255)/256, nx)
template <typename T, typename Ti>
__global__ void __launch_bounds__(256) k_refine_update(UpdateArgs<T, Ti> a) {
    pdl_begin();
    refine_update_tile(a, blockIdx.x, blockIdx.y);
}

// Device-side right-hand side: a sum of separable sine modes at the grid points.
struct SineModes {
    int n;
    double amp[64], wx[64], wy[64], wz[64];  // wx = kx*pi/Lx etc.
};

// f(i,j,k) = sum_s amp[s] sin(wx[s] x) sin(wy[s] y) sin(wz[s] z), (x,y,z) = (i,j,k)*h.  The modes
// are separable, so a block (a tile of 32 k by 8 j, marching a range of planes i) evaluates the
// sines of its k and j values once into shared memory and those of each plane once; every
// point then sums the same products in the same order as a direct evaluation would.
__global__ void __launch_bounds__(256) k_fill_sine(double* f, Geom G, double h, const SineModes m, int ichunk) {
    __shared__ double sz[64][32], sy[64][8], sx[64];
    const int tk = threadIdx.x & 31, tj = threadIdx.x >> 5;
    const int k = blockIdx.x * 32 + tk, j = blockIdx.y * 8 + tj;
    for (int q = threadIdx.x; q < m.n * 32; q += 256) {
        const int s = q >> 5, kk = blockIdx.x * 32 + (q & 31);
        sz[s][q & 31] = sin(m.wz[s] * (kk * h));
    }
    for (int q = threadIdx.x; q < m.n * 8; q += 256) {
        const int s = q >> 3, jj = blockIdx.y * 8 + (q & 7);
        sy[s][q & 7] = sin(m.wy[s] * (jj * h));
    }
    const int i0 = blockIdx.z * ichunk, i1 = min(G.nx, i0 + ichunk);
    for (int i = i0; i < i1; i++) {
        __syncthreads();  // tables ready; the previous plane's sx no longer read
        if (threadIdx.x < m.n) sx[threadIdx.x] = sin(m.wx[threadIdx.x] * (i * h));
        __syncthreads();
        if (k < G.nz && j < G.ny) {
            double acc = 0.0;
            for (int s = 0; s < m.n; s++) acc += m.amp[s] * sx[s] * sy[s][tj] * sz[s][tk];
            f[(long long)i * G.sx + (long long)j * G.sy + k] = acc;
        }
    }
}

// The reference's test problems (src/problem_definition.cpp) on the device.
__device__ __forceinline__ double prob_u(int p, double x, double y, double z) {
    switch (p) {
        case 1: return sin(3.0 * x) * sin(5.3 * y) * sin(-7.8 * z);
        case 2: return x * x * x * y * y * z;
        default: return cos(x * z * z) * sin(y * y * y);
    }
}
__device__ __forceinline__ double prob_f(int p, double x, double y, double z) {
    switch (p) {
        case 1: return -(3.0 * 3.0 + 5.3 * 5.3 + (-7.8) * (-7.8)) * sin(3.0 * x) * sin(5.3 * y) * sin(-7.8 * z);
        case 2: return 2.0 * x * x * x * z + 6.0 * x * y * y * z;
        default:
            return ((-4.0 * x * x * z * z - 9.0 * y * y * y * y - z * z * z * z) * sin(y * y * y) +
                    6.0 * y * cos(y * y * y)) * cos(x * z * z) -
                   2.0 * x * sin(x * z * z) * sin(y * y * y);
    }
}
__device__ __forceinline__ double prob_d(int p, int axis, double x, double y, double z) {
    if (p == 1) {
        if (axis == 0) return 3.0 * cos(3.0 * x) * sin(5.3 * y) * sin(-7.8 * z);
        if (axis == 1) return 5.3 * sin(3.0 * x) * cos(5.3 * y) * sin(-7.8 * z);
        return -7.8 * sin(3.0 * x) * sin(5.3 * y) * cos(-7.8 * z);
    }
    if (p == 2) {
        if (axis == 0) return 3.0 * x * x * y * y * z;
        if (axis == 1) return 2.0 * x * x * x * y * z;
        return x * x * x * y * y;
    }
    if (axis == 0) return -z * z * sin(x * z * z) * sin(y * y * y);
    if (axis == 1) return 3.0 * cos(x * z * z) * y * y * cos(y * y * y);
    return -2 * x * z * sin(x * z * z) * sin(y * y * y);
}

struct ProblemFill {
    int problem;
    double x0, y0, z0, h;
};

__global__ void __launch_bounds__(256) k_fill_problem_f(double* f, double* u, Geom G, ProblemFill pf) {
    const long long n = (long long)G.nx * G.ny * G.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % G.nz);
        const long long q = t / G.nz;
        const int j = (int)(q % G.ny);
        const int i = (int)(q / G.ny);
        const long long o = (long long)i * G.sx + (long long)j * G.sy + k;
        f[o] = prob_f(pf.problem, pf.x0 + ((double)i) * pf.h, pf.y0 + ((double)j) * pf.h, pf.z0 + ((double)k) * pf.h);
        u[o] = 0.0;
    }
}

// Boundary::init_by_fun (include/boundary.h:81-111) for one face: Dirichlet faces sample u,
// Neumann faces the derivative normal to the face (neumann.h:63-79).
__global__ void __launch_bounds__(256) k_fill_problem_face(double* g, Geom G, ProblemFill pf, int fc, int neumann) {
    int n0, n1;
    if (fc == F_EAST || fc == F_WEST) { n0 = G.ny; n1 = G.nz; }
    else if (fc == F_NORTH || fc == F_SOUTH) { n0 = G.nx; n1 = G.nz; }
    else { n0 = G.nx; n1 = G.ny; }
    const long long n = (long long)n0 * n1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t % n1), a0 = (int)(t / n1);
        double i, j, k;
        if (fc == F_EAST || fc == F_WEST) { i = fc == F_EAST ? G.nx - 1 : 0; j = a0; k = b; }
        else if (fc == F_NORTH || fc == F_SOUTH) { i = a0; j = fc == F_NORTH ? G.ny - 1 : 0; k = b; }
        else { i = a0; j = b; k = fc == F_TOP ? G.nz - 1 : 0; }
        const double x = pf.x0 + i * pf.h, y = pf.y0 + j * pf.h, z = pf.z0 + k * pf.h;
        const int axis = (fc == F_EAST || fc == F_WEST) ? 0 : (fc == F_NORTH || fc == F_SOUTH) ? 1 : 2;
        g[t] = neumann ? prob_d(pf.problem, axis, x, y, z) : prob_u(pf.problem, x, y, z);
    }
}

// Error reduction: out[0] max|u-v| (bits), out[1] sum (u-v)^2, out[2] sum v^2, out[3] max|v|.
__global__ void __launch_bounds__(256) k_u_error(const double* __restrict__ u, const double* __restrict__ v, Geom G,
                                                 Geom Gv, ProblemFill pf, unsigned long long* mx, double* sums) {
    __shared__ double red[2][8];
    const long long n = (long long)G.nx * G.ny * G.nz;
    unsigned long long m0 = 0, m1 = 0;
    double s1 = 0.0, s2 = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % G.nz);
        const long long q = t / G.nz;
        const int j = (int)(q % G.ny);
        const int i = (int)(q / G.ny);
        const double a = u[(long long)i * G.sx + (long long)j * G.sy + k];
        const double b = v ? v[(long long)i * Gv.sx + (long long)j * Gv.sy + k]
                           : prob_u(pf.problem, pf.x0 + i * pf.h, pf.y0 + j * pf.h, pf.z0 + k * pf.h);
        const double d = a - b;
        m0 = max(m0, abs_bits(d));
        m1 = max(m1, abs_bits(b));
        s1 += d * d;
        s2 += b * b;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][w] = s1;
        red[1][w] = s2;
    }
    block_max_to(m0, mx);
    block_max_to(m1, mx + 1);
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
            a += red[0][q];
            b += red[1][q];
        }
        atomicAdd(sums, a);
        atomicAdd(sums + 1, b);
    }
}

// splitmix64 (Steele, Lea, Flood 2014) as a counter-based generator.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void __launch_bounds__(256) k_fill_uniform(double* f, Geom G, unsigned long long seed, double lo, double hi) {
    const long long n = (long long)G.nx * G.ny * G.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % G.nz);
        const long long q = t / G.nz;
        const int j = (int)(q % G.ny);
        const int i = (int)(q / G.ny);
        const unsigned long long r = splitmix64(seed + (unsigned long long)t * 0x9E3779B97F4A7C15ull);
        const double u01 = (double)(r >> 11) * 0x1.0p-53;
        f[(long long)i * G.sx + (long long)j * G.sy + k] = lo + (hi - lo) * u01;
    }
}

// Dirichlet::write_to (include/dirichlet.h:50-93): one face into its boundary plane.
// Repacking between the pitched device layout and a device copy of the reference's
// halo-padded host layout (stage[off + i*hs0 + j*hs1 + k]); only shape points move, so the
// halo entries of the staging copy are neither read (TO_DEV) nor written (!TO_DEV).
template <typename T, bool TO_DEV>
__global__ void __launch_bounds__(256) k_repack(T* dev, Geom G, T* stage, long long off, long long hs0, long long hs1) {
    // launched as a programmatic dependent: wait for the previous grid (which may still be
    // writing the field being downloaded, or reading the one being uploaded)
    pdl_begin();
    const long long n = (long long)G.nx * G.ny * G.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % G.nz);
        const long long q = t / G.nz;
        const int j = (int)(q % G.ny);
        const int i = (int)(q / G.ny);
        const long long pd = (long long)i * G.sx + (long long)j * G.sy + k;
        const long long ph = off + i * hs0 + j * hs1 + k;
        if (TO_DEV) dev[pd] = stage[ph];
        else stage[ph] = dev[pd];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_write_face(T* u, Geom G, const T* __restrict__ g, int fc) {
    int n0, n1;  // face extents in its two free dimensions
    if (fc == F_EAST || fc == F_WEST) { n0 = G.ny; n1 = G.nz; }
    else if (fc == F_NORTH || fc == F_SOUTH) { n0 = G.nx; n1 = G.nz; }
    else { n0 = G.nx; n1 = G.ny; }
    const long long n = (long long)n0 * n1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t % n1), a0 = (int)(t / n1);
        int i, j, k;
        if (fc == F_EAST || fc == F_WEST) { i = fc == F_EAST ? G.nx - 1 : 0; j = a0; k = b; }
        else if (fc == F_NORTH || fc == F_SOUTH) { i = a0; j = fc == F_NORTH ? G.ny - 1 : 0; k = b; }
        else { i = a0; j = b; k = fc == F_TOP ? G.nz - 1 : 0; }
        u[(long long)i * G.sx + (long long)j * G.sy + k] = g[t];
    }
}

}  // namespace mgp
