// sc_fft.cu -- open-boundary Hockney convolution on the doubled grid.
//
// The reference (FFTPoissonSolver.cpp:337-382) zero-pads rho into the doubled
// (2n)^3 grid, multiplies its unnormalised forward transform by that of the
// mirrored integrated Green's function and transforms back with 1/(2n)^3
// (FFT.hpp:726-732, :1706).  Here the same circular convolution is computed
// with batched radix FFTs in shared memory, pruned to the non-zero octant:
//
//   A  z: real -> half spectrum, columns (x<n0, y<n1), 2 real columns per complex FFT
//   B  y: forward, input rows y<n1 only
//   C  x: forward, multiply by the real spectrum of G, inverse; input and
//         output x<n0 only
//   D  y: inverse, outputs y<n1 only
//   E  z: half spectrum -> real, 2 columns per complex FFT, outputs z<n2 only,
//         times normFact (and the cell volume and 1/(4 pi eps0) for the
//         self-field path)
//
// Spectrum layout: spec[kz][ky][kx], kx fastest, kz in [0, n2].
// The mirrored Green's function G2 is even along every axis, so its
// transform is real and is the product of three cosine (DCT-I) transforms of
// G on (n0+1)(n1+1)(n2+1) points; it is built here from G with the same FFT
// stages applied to the even extension of each line.
//
// Every kernel stages its lines global -> shared with cp.async (all copies of
// a block in flight at once, no register round trip), runs Stockham radix
// stages in shared memory and writes the pruned output.  The transform
// lengths of the common meshes (2n = 32, 64, 96, 128, 256) are template
// constants, so the stage loops unroll and the index arithmetic folds; other
// lengths take the same kernels with the length read at run time.
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <string>
#include <type_traits>
#include <vector>

#include "sc_internal.h"

namespace sc {
namespace {

template <typename T>
struct CT;
template <>
struct CT<double> {
    using type = double2;
};
template <>
struct CT<float> {
    using type = float2;
};
template <typename T>
using Cx = typename CT<T>::type;

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
    return {a.x + b.x, a.y + b.y};
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
    return {a.x - b.x, a.y - b.y};
}
// Complex product with its two fused multiply-adds written out.  The file is
// compiled without FMA contraction (-fmad=false), so every kernel that shares
// these butterflies rounds identically, whatever the surrounding code: the
// staged, register-resident and batched transforms give the same bits.
__device__ __forceinline__ float fmx(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmx(double a, double b, double c) { return fma(a, b, c); }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
    return {fmx(a.x, b.x, -(a.y * b.y)), fmx(a.x, b.y, a.y * b.x)};
}

// ---------------------------------------------------------------- cp.async
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
template <typename V>
__device__ __forceinline__ void cp_elem(V* smem, const V* gmem) {
    cp_async<(int)sizeof(V)>(smem, gmem);
}

// ---------------------------------------------------------------- plans
// Radix sequence of a length L = 2^p 3^a 5^b: radix-8 stages for the power of
// two (a remainder of 2 with an 8 becomes 4 x 4, so no radix-2 stage runs
// beside radix 8), then 3s and 5s.  nst = -1 when L has another factor.
struct RadixPlan {
    int nst;
    int r[12];
};
__host__ __device__ constexpr RadixPlan radix_plan(int L) {
    RadixPlan p{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
    if (L < 2) {
        p.nst = -1;
        return p;
    }
    int m = L, twos = 0;
    while (m % 2 == 0) {
        m /= 2;
        ++twos;
    }
    int e8 = twos / 3;
    const int rem = twos % 3;
    if (rem == 1 && e8 > 0) {
        e8 -= 1;
        p.r[p.nst++] = 4;
        p.r[p.nst++] = 4;
    } else if (rem == 1) {
        p.r[p.nst++] = 2;
    } else if (rem == 2) {
        p.r[p.nst++] = 4;
    }
    for (int i = 0; i < e8; ++i) p.r[p.nst++] = 8;
    while (m % 3 == 0 && p.nst < 12) {
        p.r[p.nst++] = 3;
        m /= 3;
    }
    while (m % 5 == 0 && p.nst < 12) {
        p.r[p.nst++] = 5;
        m /= 5;
    }
    if (m != 1) p.nst = -1;
    return p;
}
__host__ __device__ constexpr int min_radix(int L) {
    const RadixPlan p = radix_plan(L);
    int r = 16;
    for (int i = 0; i < p.nst; ++i) r = p.r[i] < r ? p.r[i] : r;
    return r;
}
// Complex transforms per block for a template length: the widest stage
// (L / min radix butterflies per transform) fills at most 256 threads, and
// at most 16 transforms share a block.  Length 0 (read at run time): 16.
__host__ __device__ constexpr int cols_for(int LT) {
    if (LT == 0) return 16;
    const int per = LT / min_radix(LT);
    int nc = 256 / per;
    if (nc > 16) nc = 16;
    if (nc < 1) nc = 1;
    return nc;
}
__host__ __device__ constexpr int threads_for(int LT) {
    if (LT == 0) return 256;
    const int t = cols_for(LT) * (LT / min_radix(LT));
    return t < 32 ? 32 : t;
}

// ---------------------------------------------------------------- butterflies
// R-point DFT in registers; forward uses exp(-2 pi i / R).
template <typename T, int R, bool INV>
__device__ __forceinline__ void dft(Cx<T>* v) {
    using C = Cx<T>;
    if constexpr (R == 2) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        C t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        if constexpr (!INV) {
            v[1] = C{t1.x + t3.y, t1.y - t3.x};
            v[3] = C{t1.x - t3.y, t1.y + t3.x};
        } else {
            v[1] = C{t1.x - t3.y, t1.y + t3.x};
            v[3] = C{t1.x + t3.y, t1.y - t3.x};
        }
    } else if constexpr (R == 3) {
        const T s = INV ? (T)0.86602540378443864676 : (T)-0.86602540378443864676;
        C t1 = cadd(v[1], v[2]);
        C d = csub(v[1], v[2]);
        C t2 = C{v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y};
        v[0] = cadd(v[0], t1);
        v[1] = C{t2.x - s * d.y, t2.y + s * d.x};
        v[2] = C{t2.x + s * d.y, t2.y - s * d.x};
    } else if constexpr (R == 8) {
        // 2 x 4: a_k = x_k + x_{k+4}, b_k = (x_k - x_{k+4}) W8^k; X_{2m} = DFT4(a), X_{2m+1} = DFT4(b)
        const T h = (T)0.70710678118654752440;
        C a[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            a[k] = cadd(v[k], v[k + 4]);
            b[k] = csub(v[k], v[k + 4]);
        }
        // W8^1 = (1 - i)/sqrt2 (forward), W8^2 = -i, W8^3 = -(1 + i)/sqrt2; conjugates for the inverse
        if constexpr (!INV) {
            b[1] = C{h * (b[1].x + b[1].y), h * (b[1].y - b[1].x)};
            b[2] = C{b[2].y, -b[2].x};
            b[3] = C{h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y)};
        } else {
            b[1] = C{h * (b[1].x - b[1].y), h * (b[1].y + b[1].x)};
            b[2] = C{-b[2].y, b[2].x};
            b[3] = C{-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y)};
        }
        dft<T, 4, INV>(a);
        dft<T, 4, INV>(b);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            v[2 * m] = a[m];
            v[2 * m + 1] = b[m];
        }
    } else if constexpr (R == 5) {
        const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
        const T s1 = INV ? (T)0.95105651629515357212 : (T)-0.95105651629515357212;
        const T s2 = INV ? (T)0.58778525229247312917 : (T)-0.58778525229247312917;
        C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
        C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
        C x0 = v[0];
        C r1 = C{x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y};
        C r2 = C{x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y};
        C i1 = C{s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y};
        C i2 = C{s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y};
        v[0] = C{x0.x + a1.x + a2.x, x0.y + a1.y + a2.y};
        v[1] = C{r1.x - i1.y, r1.y + i1.x};
        v[4] = C{r1.x + i1.y, r1.y - i1.x};
        v[2] = C{r2.x - i2.y, r2.y + i2.x};
        v[3] = C{r2.x + i2.y, r2.y - i2.x};
    }
}

// Shared-memory position of element i of a column: one empty slot after every
// 8 elements.  The first Stockham stages write with strides of R elements
// (R = 4 or 8, i.e. 64 or 128 bytes of complex double), which would put a
// warp's stores into one or two bank groups; the skew spreads them over all.
__host__ __device__ constexpr int sk(int i) { return i + (i >> 3); }

// R-point DFT of inputs whose upper half v[R/2 .. R-1] is zero (the
// zero-padded half of a forward transform's first stage).
template <typename T, int R, bool INV>
__device__ __forceinline__ void dft_half(Cx<T>* v) {
    using C = Cx<T>;
    if constexpr (R == 2) {
        v[1] = v[0];
    } else if constexpr (R == 4) {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[2] = csub(a, b);
        if constexpr (!INV) {
            v[1] = C{a.x + b.y, a.y - b.x};
            v[3] = C{a.x - b.y, a.y + b.x};
        } else {
            v[1] = C{a.x - b.y, a.y + b.x};
            v[3] = C{a.x + b.y, a.y - b.x};
        }
    } else {
        static_assert(R == 8, "half-input DFT for radix 2, 4, 8");
        const T h = (T)0.70710678118654752440;
        C a[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) a[k] = b[k] = v[k];
        if constexpr (!INV) {
            b[1] = C{h * (b[1].x + b[1].y), h * (b[1].y - b[1].x)};
            b[2] = C{b[2].y, -b[2].x};
            b[3] = C{h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y)};
        } else {
            b[1] = C{h * (b[1].x - b[1].y), h * (b[1].y + b[1].x)};
            b[2] = C{-b[2].y, b[2].x};
            b[3] = C{-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y)};
        }
        dft<T, 4, INV>(a);
        dft<T, 4, INV>(b);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            v[2 * m] = a[m];
            v[2 * m + 1] = b[m];
        }
    }
}

// One Stockham autosort butterfly (radix R): butterfly j of a column reads
// element j + r nb, r < R, applies the twiddles W^(r k step), k = j mod Ns,
// and writes element (j / Ns) Ns R + k + r Ns (positions through sk()).
// NZ < R: inputs r >= NZ are known zeros (NZ = R/2 only); NO < R: only
// outputs r < NO are needed; FIRST: Ns = 1, all twiddles are 1.
template <typename T, int R, bool INV, int NZ = R, int NO = R, bool FIRST = false>
__device__ __forceinline__ void butterfly(const Cx<T>* __restrict__ src, Cx<T>* __restrict__ dst, int j, int nb, int Ns,
                                          int step, const Cx<T>* __restrict__ tw) {
    using C = Cx<T>;
    static_assert(NZ == R || (2 * NZ == R && FIRST), "zero inputs only in a first stage");
    C v[R];
#pragma unroll
    for (int r = 0; r < NZ; ++r) v[r] = src[sk(j + r * nb)];
    const int k = FIRST ? 0 : j % Ns;
    if constexpr (!FIRST) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
            C t = tw[r * k * step];
            if (INV) t.y = -t.y;
            v[r] = cmul(v[r], t);
        }
    }
    if constexpr (NZ == R)
        dft<T, R, INV>(v);
    else
        dft_half<T, R, INV>(v);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < NO; ++r) dst[sk(base + r * Ns)] = v[r];
}

// Column stride: the L skewed elements (sk(L - 1) < L + L/8) plus one, so
// that the columns of a block also start in different banks.
__host__ __device__ constexpr int col_stride(int L) { return L + (L >> 3) + 1; }

// Pruning of a transform whose length is a template constant:
//   kPruneNone  full transform;
//   kPruneIn    the upper half of the input is zero (forward transforms of
//               the zero-padded doubled grid): the first stage reads half;
//   kPruneOut   only the lower half of the output is used (inverse
//               transforms back to the physical octant): the last stage
//               writes half.
constexpr int kPruneNone = 0, kPruneIn = 1, kPruneOut = 2;

// compile-time stage: length L, Ns, NC columns, NT threads
template <typename T, int R, bool INV, int L, int NS, int NC, int NT, int NZ, int NO>
__device__ __forceinline__ void stage_c(const Cx<T>* in, Cx<T>* out, const Cx<T>* tw) {
    constexpr int NB = L / R;
    constexpr int STEP = L / (NS * R);
    constexpr int CS = col_stride(L);
#pragma unroll
    for (int w0 = 0; w0 < NC * NB; w0 += NT) {
        const int w = w0 + (int)threadIdx.x;
        if ((NC * NB) % NT != 0 && w >= NC * NB) break;
        const int col = w / NB;
        const int j = w - col * NB;
        butterfly<T, R, INV, NZ, NO, NS == 1>(in + col * CS, out + col * CS, j, NB, NS, STEP, tw);
    }
}

template <typename T, bool INV, int L, int S, int NS, int NC, int NT, int PR>
__device__ __forceinline__ Cx<T>* stages_c(Cx<T>* a, Cx<T>* b, const Cx<T>* tw) {
    constexpr RadixPlan P = radix_plan(L);
    if constexpr (S == P.nst) {
        return a;
    } else {
        constexpr int R = P.r[S];
        constexpr bool even = R % 2 == 0;
        constexpr int NZ = (PR == kPruneIn && S == 0 && even && R <= 8) ? R / 2 : R;
        constexpr int NO = (PR == kPruneOut && S == P.nst - 1 && even) ? R / 2 : R;
        stage_c<T, R, INV, L, NS, NC, NT, NZ, NO>(a, b, tw);
        __syncthreads();
        return stages_c<T, INV, L, S + 1, NS * R, NC, NT, PR>(b, a, tw);
    }
}

// run-time stage (lengths without a template instance)
template <typename T, int R, bool INV>
__device__ __forceinline__ void stage_r(const Cx<T>* in, Cx<T>* out, int L, int Ns, int ncols, const Cx<T>* tw) {
    const int nb = L / R;
    const int step = L / (Ns * R);
    const int cs = col_stride(L);
    for (int w = threadIdx.x; w < ncols * nb; w += blockDim.x) {
        const int col = w / nb;
        const int j = w - col * nb;
        butterfly<T, R, INV>(in + col * cs, out + col * cs, j, nb, Ns, step, tw);
    }
}

// Complex FFT of NC columns (element i of column col at buf[col * col_stride(L) + sk(i)]); returns the buffer holding
// the result (buf or tmp).  The caller synchronises before the call.
// With a template length the transform is pruned as PR says (the caller
// then stages only the nonzero half, or reads only the lower half); with a
// run-time length it is always full.
template <typename T, bool INV, int LT, int NC, int NT, int PR = kPruneNone>
__device__ __forceinline__ Cx<T>* block_fft(Cx<T>* buf, Cx<T>* tmp, const FftPlan& pl, const Cx<T>* tw) {
    if constexpr (LT > 0) {
        return stages_c<T, INV, LT, 0, 1, NC, NT, PR>(buf, tmp, tw);
    } else {
        int Ns = 1;
        Cx<T>* a = buf;
        Cx<T>* b = tmp;
        for (int s = 0; s < pl.nst; ++s) {
            const int R = pl.r[s];
            if (R == 8)
                stage_r<T, 8, INV>(a, b, pl.L, Ns, NC, tw);
            else if (R == 4)
                stage_r<T, 4, INV>(a, b, pl.L, Ns, NC, tw);
            else if (R == 2)
                stage_r<T, 2, INV>(a, b, pl.L, Ns, NC, tw);
            else if (R == 3)
                stage_r<T, 3, INV>(a, b, pl.L, Ns, NC, tw);
            else
                stage_r<T, 5, INV>(a, b, pl.L, Ns, NC, tw);
            __syncthreads();
            Cx<T>* t = a;
            a = b;
            b = t;
            Ns *= R;
        }
        return a;
    }
}

template <typename V, int NT>
__device__ __forceinline__ void stage_twiddles(V* dst, const V* __restrict__ src, int L) {
    for (int e = threadIdx.x; e < L; e += NT) cp_elem(dst + e, src + e);
}

// elements of one tile: twiddles (L), buf and tmp (NC col_stride(L) + 2 NC each)
__host__ __device__ constexpr size_t tile_elems(int L, int nc) {
    return (size_t)L + 2 * ((size_t)nc * col_stride(L) + 2 * nc);
}

// ---------------------------------------------------------------- pass A
// 2 NC real columns (x) of one y per block, packed two per complex FFT.
// FULL: the z transform covers the data without zero padding (periodic z,
// L2 = n2); otherwise L2 = 2 n2 and the upper half is zero.  The half
// spectrum has L2/2 + 1 entries either way.
template <typename T, int LT, int NC, int NT, bool FULL = false>
__device__ __forceinline__ void fft_z_r2c_body(const T* __restrict__ rho, Cx<T>* __restrict__ spec, int n0, int n1, int n2,
                                               int L0, int L1, const FftPlan& pz, const Cx<T>* __restrict__ twz, int bx,
                                               int by) {
    using C = Cx<T>;
    constexpr int RC = 2 * NC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L2 = LT > 0 ? LT : pz.L;
    const int CS = col_stride(L2);
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + L2;
    C* tmp = buf + NC * CS + RC;
    stage_twiddles<C, NT>(tw, twz, L2);
    const int y = by;
    const int x0 = bx * RC;
    for (int e = threadIdx.x; e < RC * (LT > 0 ? n2 : L2); e += NT) {  // the zero half is not staged when pruned
        const int xi = e % RC, z = e / RC;
        const int x = x0 + xi;
        T* slot = reinterpret_cast<T*>(&buf[(xi >> 1) * CS + sk(z)]) + (xi & 1);
        if (z < n2 && x < n0)
            cp_elem(slot, &rho[((size_t)z * n1 + y) * n0 + x]);
        else
            *slot = (T)0;
    }
    cp_async_wait_all();
    __syncthreads();
    const C* out = block_fft<T, false, LT, NC, NT, FULL ? kPruneNone : kPruneIn>(buf, tmp, pz, tw);
    const int K = L2 / 2;
    for (int e = threadIdx.x; e < RC * (K + 1); e += NT) {
        const int xi = e % RC, k = e / RC;
        const int x = x0 + xi;
        if (x >= n0) continue;
        const int q = xi >> 1;
        const C Z = out[q * CS + sk(k)];
        const C Zm = out[q * CS + sk(k == 0 ? 0 : L2 - k)];
        C r;
        if ((xi & 1) == 0)
            r = C{(T)0.5 * (Z.x + Zm.x), (T)0.5 * (Z.y - Zm.y)};
        else
            r = C{(T)0.5 * (Z.y + Zm.y), (T)-0.5 * (Z.x - Zm.x)};
        spec[((size_t)k * L1 + y) * L0 + x] = r;
    }
}
template <typename T, int LT, int NC, int NT, bool FULL = false>
__global__ void __launch_bounds__(NT, 1024 / NT) k_fft_z_r2c(const T* __restrict__ rho, Cx<T>* __restrict__ spec, int n0, int n1, int n2,
                                                  int L0, int L1, FftPlan pz, const Cx<T>* __restrict__ twz) {
    fft_z_r2c_body<T, LT, NC, NT, FULL>(rho, spec, n0, n1, n2, L0, L1, pz, twz, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------- pass B / D
// NC x-columns of one kz plane per block; rows y < n_in in, y < n_out out.
template <typename T, bool INV, int LT, int NC, int NT>
__device__ __forceinline__ void fft_y_body(Cx<T>* __restrict__ spec, int n0, int L0, int n_in, int n_out, const FftPlan& py,
                                           const Cx<T>* __restrict__ twy, int bx, int by) {
    using C = Cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L1 = LT > 0 ? LT : py.L;
    const int CS = col_stride(L1);
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + L1;
    C* tmp = buf + NC * CS + 2 * NC;
    stage_twiddles<C, NT>(tw, twy, L1);
    const int kz = by;
    const int x0 = bx * NC;
    C* plane = spec + (size_t)kz * L1 * L0;
    for (int e = threadIdx.x; e < NC * ((LT > 0 && !INV) ? n_in : L1); e += NT) {
        const int xi = e % NC, yy = e / NC;
        const int x = x0 + xi;
        C* slot = &buf[xi * CS + sk(yy)];
        if (yy < n_in && x < n0)
            cp_elem(slot, &plane[(size_t)yy * L0 + x]);
        else
            *slot = C{(T)0, (T)0};
    }
    cp_async_wait_all();
    __syncthreads();
    const C* out = block_fft<T, INV, LT, NC, NT, INV ? kPruneOut : kPruneIn>(buf, tmp, py, tw);
    for (int e = threadIdx.x; e < NC * n_out; e += NT) {
        const int xi = e % NC, yy = e / NC;
        const int x = x0 + xi;
        if (x < n0) plane[(size_t)yy * L0 + x] = out[xi * CS + sk(yy)];
    }
}
template <typename T, bool INV, int LT, int NC, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_fft_y(Cx<T>* __restrict__ spec, int n0, int L0, int n_in, int n_out, FftPlan py,
                                              const Cx<T>* __restrict__ twy) {
    fft_y_body<T, INV, LT, NC, NT>(spec, n0, L0, n_in, n_out, py, twy, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------- pass C
// The forward transform and the multiplication run in TI, the inverse in TO.
// The mixed form takes TI = float, TO = double: rounding in the forward half
// is white noise in the spectrum, which the derivative of phi does not
// amplify, while rounding after the multiplication would be noise relative
// to phi itself and is kept at FP64.  `in` and `out` alias in the plain form;
// every block reads its rows before it writes them.
//
// CG: ghat holds complex values (the image charge's shifted G is not even in
// z, FFTPoissonSolver.cpp:316); the product is the complex one.
template <typename TI, typename TO, int LT, int NC, int NT, bool CG = false>
__device__ __forceinline__ void fft_x_conv_body(const Cx<TI>* in, Cx<TO>* out, const TI* __restrict__ ghat, int n0, int n1,
                                                int L1, int rows, const FftPlan& px, const Cx<TI>* __restrict__ twi,
                                                const Cx<TO>* __restrict__ two, int bx) {
    using CI = Cx<TI>;
    using CO = Cx<TO>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L0 = LT > 0 ? LT : px.L;
    const int CS = col_stride(L0);
    CO* tw_o = reinterpret_cast<CO*>(smem_raw);
    CI* tw_i = reinterpret_cast<CI*>(tw_o + L0);
    CO* bufo = reinterpret_cast<CO*>(tw_i + L0);
    CO* tmpo = bufo + NC * CS;
    stage_twiddles<CO, NT>(tw_o, two, L0);
    stage_twiddles<CI, NT>(tw_i, twi, L0);
    CI* bufi = reinterpret_cast<CI*>(bufo);
    CI* tmpi = reinterpret_cast<CI*>(tmpo);
    const int r0 = bx * NC;
    const int xs = LT > 0 ? n0 : L0;  // staged length: the zero half is not staged when pruned
    for (int e = threadIdx.x; e < NC * xs; e += NT) {
        const int ri = e / xs, x = e - ri * xs;
        const int r = r0 + ri;
        CI* slot = &bufi[ri * CS + sk(x)];
        if (r < rows && x < n0)
            cp_elem(slot, &in[(size_t)r * L0 + x]);
        else
            *slot = CI{(TI)0, (TI)0};
    }
    cp_async_wait_all();
    __syncthreads();
    const CI* f = block_fft<TI, false, LT, NC, NT, kPruneIn>(bufi, tmpi, px, tw_i);
    CO* g = (f == bufi) ? tmpo : bufo;
    CO* h = (f == bufi) ? bufo : tmpo;
    for (int e = threadIdx.x; e < NC * L0; e += NT) {
        const int ri = e / L0, kx = e - ri * L0;
        const int r = r0 + ri;
        if (r >= rows) continue;
        const int kz = r / L1;
        const int ky = r - kz * L1;
        const int gy = ky <= n1 ? ky : L1 - ky;
        const int gx = kx <= n0 ? kx : L0 - kx;
        const size_t gi = ((size_t)kz * (n1 + 1) + gy) * (n0 + 1) + gx;
        const CI v = f[ri * CS + sk(kx)];
        if constexpr (CG) {
            const CI gc = reinterpret_cast<const CI*>(ghat)[gi];
            g[ri * CS + sk(kx)] = CO{(TO)(v.x * gc.x - v.y * gc.y), (TO)(v.x * gc.y + v.y * gc.x)};
        } else {
            const TI gv = ghat[gi];
            g[ri * CS + sk(kx)] = CO{(TO)(v.x * gv), (TO)(v.y * gv)};
        }
    }
    __syncthreads();
    const CO* o = block_fft<TO, true, LT, NC, NT, kPruneOut>(g, h, px, tw_o);
    for (int e = threadIdx.x; e < NC * n0; e += NT) {
        const int ri = e / n0, x = e - ri * n0;
        const int r = r0 + ri;
        if (r < rows) out[(size_t)r * L0 + x] = o[ri * CS + sk(x)];
    }
}
template <typename TI, typename TO, int LT, int NC, int NT, bool CG = false>
__global__ void __launch_bounds__(NT, 1024 / NT) k_fft_x_conv(const Cx<TI>* in, Cx<TO>* out, const TI* __restrict__ ghat, int n0, int n1,
                                                   int L1, int rows, FftPlan px, const Cx<TI>* __restrict__ twi,
                                                   const Cx<TO>* __restrict__ two) {
    fft_x_conv_body<TI, TO, LT, NC, NT, CG>(in, out, ghat, n0, n1, L1, rows, px, twi, two, blockIdx.x);
}

// ---------------------------------------------------------------- lines in registers
// The same Stockham transform of a 64-, 128- or 256-point line (plans 8 8;
// 4 4 8; 4 8 8: the same butterflies, twiddles and operation order as
// block_fft, so the same bits), computed by 8 threads of one warp with the
// data in registers: thread a holds elements a + 8m (m < L/8).  Those are
// exactly the inputs of the first stage's butterflies a + 8q; for 128 and 256
// points their outputs are in turn the inputs of the second stage's
// butterflies 4a + k, which leave elements (L/8)a .. (L/8)a + L/8 - 1 in the
// thread.  One exchange through the line's shared buffer (element p at
// p + p/(L/8): the 8 threads' accesses fall in distinct banks) gives thread a
// the inputs of the last stage's butterflies a + 8s, whose outputs are the
// elements a + 8m again.  No block barrier: the 8 threads of a line are a
// quarter of a warp.
template <int L>
struct LineGeo {
    static constexpr int M = L / 8;           // elements per thread
    static constexpr int BUF = L + 8;         // exchange buffer elements of a line
    static constexpr int LINES = L >= 256 ? 8 : 16;  // lines per block
    static constexpr int NT = 8 * LINES;
};
template <int L>
__device__ __forceinline__ int xidx(int p) {
    return p + p / (L / 8);
}

// BLOCK: the 8 threads of a line sit in different warps (the y passes, whose
// lanes run along x for coalesced columns); the exchange then waits for the
// whole block.
template <bool BLOCK>
__device__ __forceinline__ void line_sync() {
    if constexpr (BLOCK)
        __syncthreads();
    else
        __syncwarp();
}

template <typename T, bool INV, bool HALF_IN, int L, bool BLOCK = false>
__device__ __forceinline__ void line_fft(Cx<T> (&v)[L / 8], int a, Cx<T>* xs, const Cx<T>* __restrict__ tw) {
    using C = Cx<T>;
    constexpr int M = L / 8;
    C o[M];  // elements M a + i after the stages before the exchange
    if constexpr (L == 64) {
        // stage 1: radix 8, Ns = 1; butterfly a reads elements a + 8r
        C u[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) u[r] = v[r];
        if constexpr (HALF_IN)
            dft_half<T, 8, INV>(u);
        else
            dft<T, 8, INV>(u);
#pragma unroll
        for (int r = 0; r < 8; ++r) o[r] = u[r];
    } else {
        constexpr int R2 = L == 128 ? 4 : 8;   // second-stage radix
        constexpr int Q = M / 4;                // first-stage butterflies per thread
        C w[Q][4];
        // stage 1: radix 4, Ns = 1; butterfly a + 8q reads elements a + 8q + (L/4) r
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            C u[4];
            u[0] = v[q];
            u[1] = v[q + Q];
            if constexpr (HALF_IN) {
                dft_half<T, 4, INV>(u);
            } else {
                u[2] = v[q + 2 * Q];
                u[3] = v[q + 3 * Q];
                dft<T, 4, INV>(u);
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) w[q][r] = u[r];
        }
        // stage 2: radix R2, Ns = 4, step L / (4 R2) = 8; butterfly 4a + k
        // reads the first stage's outputs 4a + k + (L/R2) r = output k of
        // butterfly a + 8r, and writes elements M a + k + 4r
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            C u[R2];
#pragma unroll
            for (int r = 0; r < R2; ++r) u[r] = w[r][k];
#pragma unroll
            for (int r = 1; r < R2; ++r) {
                C t = __ldg(&tw[r * k * 8]);
                if (INV) t.y = -t.y;
                u[r] = cmul(u[r], t);
            }
            dft<T, R2, INV>(u);
#pragma unroll
            for (int r = 0; r < R2; ++r) o[k + 4 * r] = u[r];
        }
    }
#pragma unroll
    for (int i = 0; i < M; ++i) xs[xidx<L>(M * a + i)] = o[i];
    line_sync<BLOCK>();
    // last stage: radix 8, Ns = M, step 1; butterfly j = a + 8s reads
    // elements j + M r and writes them back in place
#pragma unroll
    for (int s2 = 0; s2 < M / 8; ++s2) {
        const int j = a + 8 * s2;
        C u[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) u[r] = xs[xidx<L>(j + M * r)];
#pragma unroll
        for (int r = 1; r < 8; ++r) {
            C t = __ldg(&tw[r * j]);
            if (INV) t.y = -t.y;
            u[r] = cmul(u[r], t);
        }
        dft<T, 8, INV>(u);
#pragma unroll
        for (int r = 0; r < 8; ++r) v[s2 + (M / 8) * r] = u[r];  // element j + M r = a + 8 (s2 + (M/8) r)
    }
    line_sync<BLOCK>();  // the buffer is free again
}

// Pass C on rows of L = 2 n0 points: 8 threads per row.  The forward
// transform leaves each thread the spectrum at a + 8m, exactly the inputs
// the inverse transform's first stages need from it.
template <typename TI, typename TO, bool CG, int L>
__device__ __forceinline__ void fft_x_conv_lines_body(const Cx<TI>* in, Cx<TO>* out, const TI* __restrict__ ghat, int n0,
                                                      int n1, int L1, int rows, const Cx<TI>* __restrict__ twi,
                                                      const Cx<TO>* __restrict__ two, int blk) {
    using CI = Cx<TI>;
    using CO = Cx<TO>;
    using G = LineGeo<L>;
    constexpr int M = G::M;
    __shared__ __align__(16) CO xbuf[G::LINES][G::BUF];
    const int li = threadIdx.x >> 3, a = threadIdx.x & 7;
    const int r = blk * G::LINES + li;
    const bool live = r < rows;
    CI v[M];
#pragma unroll
    for (int m = 0; m < M; ++m)
        v[m] = (live && m < M / 2) ? in[(size_t)r * L + a + 8 * m] : CI{(TI)0, (TI)0};
    const int kz = live ? r / L1 : 0;
    const int ky = live ? r - kz * L1 : 0;
    const int gy = ky <= n1 ? ky : L1 - ky;
    const size_t grow = ((size_t)kz * (n1 + 1) + gy) * (n0 + 1);
    // the row of G's spectrum is fetched before the forward transform, so its
    // latency hides behind the transform
    using GV = typename std::conditional<CG, CI, TI>::type;
    GV g[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int kx = a + 8 * m;
        const int gx = kx <= n0 ? kx : L - kx;
        g[m] = live ? reinterpret_cast<const GV*>(ghat)[grow + gx] : GV{};
    }
    line_fft<TI, false, true, L>(v, a, reinterpret_cast<CI*>(xbuf[li]), twi);
    CO w[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const CI f = v[m];
        if constexpr (CG) {
            const CI gc = g[m];
            w[m] = CO{(TO)(f.x * gc.x - f.y * gc.y), (TO)(f.x * gc.y + f.y * gc.x)};
        } else {
            const TI gv = g[m];
            w[m] = CO{(TO)(f.x * gv), (TO)(f.y * gv)};
        }
    }
    line_fft<TO, true, false, L>(w, a, xbuf[li], two);
    if (!live) return;
#pragma unroll
    for (int m = 0; m < M / 2; ++m) out[(size_t)r * L + a + 8 * m] = w[m];  // x < n0
}

template <typename TI, typename TO, bool CG, int L>
__global__ void __launch_bounds__(LineGeo<L>::NT) k_fft_x_conv_lines(const Cx<TI>* in, Cx<TO>* out,
                                                                   const TI* __restrict__ ghat, int n0, int n1, int L1,
                                                                   int rows, const Cx<TI>* __restrict__ twi,
                                                                   const Cx<TO>* __restrict__ two) {
    fft_x_conv_lines_body<TI, TO, CG, L>(in, out, ghat, n0, n1, L1, rows, twi, two, blockIdx.x);
}

// Passes B (forward, inputs y < L/2) and D (inverse, outputs y < L/2) on
// columns of L points along y: 8 threads per column (in different warps),
// consecutive x of one plane per block.
template <typename T, bool INV, int L>
__device__ __forceinline__ void fft_y_lines_body(Cx<T>* __restrict__ spec, int n0, int L0, int planes,
                                                 const Cx<T>* __restrict__ twy, int bx, int kz) {
    using C = Cx<T>;
    using G = LineGeo<L>;
    constexpr int M = G::M;
    // lanes run along x (thread li + LINES a: column li, part a), so a warp
    // reads and writes whole rows of consecutive columns; the line buffers
    // are G::BUF + 1 apart, so the lines of one access fall in distinct banks
    __shared__ __align__(16) C xbuf[G::LINES][G::BUF + 1];
    const int li = threadIdx.x % G::LINES, a = threadIdx.x / G::LINES;
    const int x = bx * G::LINES + li;
    const bool live = kz < planes && x < n0;
    C* col = spec + (size_t)kz * L * L0 + (live ? x : 0);
    C v[M];
#pragma unroll
    for (int m = 0; m < M; ++m)
        v[m] = (live && (INV || m < M / 2)) ? col[(size_t)(a + 8 * m) * L0] : C{(T)0, (T)0};
    line_fft<T, INV, !INV, L, true>(v, a, xbuf[li], twy);
    if (!live) return;
    constexpr int MO = INV ? M / 2 : M;  // D keeps y < L/2
#pragma unroll
    for (int m = 0; m < MO; ++m) col[(size_t)(a + 8 * m) * L0] = v[m];
}

template <typename T, bool INV, int L>
__global__ void __launch_bounds__(LineGeo<L>::NT) k_fft_y_lines(Cx<T>* __restrict__ spec, int n0, int L0, int planes,
                                                              const Cx<T>* __restrict__ twy) {
    fft_y_lines_body<T, INV, L>(spec, n0, L0, planes, twy, blockIdx.x, blockIdx.y);
}

// Pass A on z lines of L = 2 n2 points: two real columns (x, x + 1) of one y
// per complex line, 8 threads per line with the lanes along x (consecutive
// column pairs, so a warp reads and writes whole rows) and block-level
// exchanges.  The two half spectra need Z[k] and Z[L - k], which sit in
// different threads: the transformed line goes through its buffer once more.
template <typename T, int L>
__global__ void __launch_bounds__(LineGeo<L>::NT) k_fft_z_r2c_lines(const T* __restrict__ rho, Cx<T>* __restrict__ spec,
                                                                  int n0, int n1, int L0, int L1,
                                                                  const Cx<T>* __restrict__ twz) {
    using C = Cx<T>;
    using G = LineGeo<L>;
    constexpr int M = G::M, K = L / 2;
    __shared__ __align__(16) C xbuf[G::LINES][G::BUF + 1];
    const int li = threadIdx.x % G::LINES, a = threadIdx.x / G::LINES;
    const int np = (n0 + 1) / 2;
    const int line = blockIdx.x * G::LINES + li;
    const int y = line / np, x = 2 * (line - y * np);
    const bool live = y < n1;
    const bool odd = live && x + 1 < n0;
    C v[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        v[m] = C{(T)0, (T)0};
        if (live && m < M / 2) {
            const T* p = rho + ((size_t)(a + 8 * m) * n1 + y) * n0 + x;
            v[m].x = p[0];
            if (odd) v[m].y = p[1];
        }
    }
    C* xs = xbuf[li];
    line_fft<T, false, true, L, true>(v, a, xs, twz);
#pragma unroll
    for (int m = 0; m < M; ++m) xs[xidx<L>(a + 8 * m)] = v[m];
    __syncthreads();
    if (!live) return;
#pragma unroll
    for (int m = 0; m <= M / 2; ++m) {
        const int k = a + 8 * m;
        if (k > K) break;
        const C Z = xs[xidx<L>(k)];
        const C Zm = xs[xidx<L>(k == 0 ? 0 : L - k)];
        C* dst = spec + ((size_t)k * L1 + y) * L0 + x;
        dst[0] = C{(T)0.5 * (Z.x + Zm.x), (T)0.5 * (Z.y - Zm.y)};
        if (odd) dst[1] = C{(T)0.5 * (Z.y + Zm.y), (T)-0.5 * (Z.x - Zm.x)};
    }
}

// ---------------------------------------------------------------- pass E
// FLIP: the image potential is read back with z flipped,
// rho[i][j][k] = rho2[i][j][n2 - k - 1] (FFTPoissonSolver.cpp:322-326).
// FULL: all L2 = n2 outputs of an unpadded (periodic) z transform.
template <typename T, bool SELF, int LT, int NC, int NT, bool FLIP = false, bool FULL = false>
__device__ __forceinline__ void fft_z_c2r_body(const Cx<T>* __restrict__ spec, double* __restrict__ phi, int n0, int n1,
                                               int n2, int L0, int L1, const FftPlan& pz, const Cx<T>* __restrict__ twz,
                                               const StepState* __restrict__ st, double normFact, double coupling, int bx,
                                               int by) {
    using C = Cx<T>;
    constexpr int RC = 2 * NC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L2 = LT > 0 ? LT : pz.L;
    const int CS = col_stride(L2);
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + L2;
    C* tmp = buf + NC * CS + RC;
    stage_twiddles<C, NT>(tw, twz, L2);
    const int y = by;
    const int x0 = bx * RC;
    // the half spectra of the 2 NC columns in tmp: [xi][k], k <= K = L2 / 2
    const int K = L2 / 2;
    for (int e = threadIdx.x; e < RC * (K + 1); e += NT) {
        const int xi = e % RC, k = e / RC;
        const int x = x0 + xi;
        C* slot = &tmp[xi * (K + 1) + k];
        if (x < n0)
            cp_elem(slot, &spec[((size_t)k * L1 + y) * L0 + x]);
        else
            *slot = C{(T)0, (T)0};
    }
    cp_async_wait_all();
    __syncthreads();
    for (int e = threadIdx.x; e < NC * L2; e += NT) {
        const int q = e / L2, k = e - q * L2;
        const C* A = tmp + (2 * q) * (K + 1);
        const C* B = tmp + (2 * q + 1) * (K + 1);
        C z;
        if (k <= K) {
            C a = A[k], b = B[k];
            if (k == 0 || k == K) {  // the half-complex format holds no imaginary part there
                a.y = (T)0;
                b.y = (T)0;
            }
            z = C{a.x - b.y, a.y + b.x};
        } else {
            const C a = A[L2 - k], b = B[L2 - k];
            z = C{a.x + b.y, b.x - a.y};
        }
        buf[q * CS + sk(k)] = z;
    }
    __syncthreads();
    const C* out = block_fft<T, true, LT, NC, NT, FULL ? kPruneNone : kPruneOut>(buf, tmp, pz, tw);
    const double hvol = SELF ? st->hvol : 1.0;
    for (int e = threadIdx.x; e < RC * n2; e += NT) {
        const int xi = e % RC, zz = e / RC;
        const int x = x0 + xi;
        if (x >= n0) continue;
        const C v = out[(xi >> 1) * CS + sk(zz)];
        double r = (double)((xi & 1) ? v.y : v.x);
        r = r * normFact;
        if (SELF) {
            r = r * hvol;
            r = r * coupling;
        }
        phi[((size_t)(FLIP ? n2 - 1 - zz : zz) * n1 + y) * n0 + x] = r;
    }
}
template <typename T, bool SELF, int LT, int NC, int NT, bool FLIP = false, bool FULL = false>
__global__ void __launch_bounds__(NT, 1024 / NT) k_fft_z_c2r(const Cx<T>* __restrict__ spec, double* __restrict__ phi, int n0, int n1,
                                                  int n2, int L0, int L1, FftPlan pz, const Cx<T>* __restrict__ twz,
                                                  const StepState* __restrict__ st, double normFact, double coupling) {
    fft_z_c2r_body<T, SELF, LT, NC, NT, FLIP, FULL>(spec, phi, n0, n1, n2, L0, L1, pz, twz, st, normFact, coupling,
                                                    blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------- G spectrum
// Cosine transform of every line along one axis: Y[m] = sum over the even
// extension (length L = 2(len-1)) of g, m in [0, len-1].  Lines are addressed
// as in[b * sb + o * so + e * se]; 2 NC lines per block (two per complex FFT).
// FROM_TMP (the z lines, b = x, o = y, e = z): in is the IGF antiderivative
// on the (t0 = n0+2) x (t1 = n1+2) grid and each element of G is formed from
// it as it is staged (igf_G_at), so G itself is never stored.
template <typename TO, int LT, int NC, int NT, bool FROM_TMP = false>
__device__ __forceinline__ void dct_lines_body(const double* __restrict__ in, TO* __restrict__ out, int len, int nb,
                                               long long sb, long long so, long long se, const FftPlan& pl,
                                               const double2* __restrict__ twd, int bx, int by, int t0 = 0,
                                               int t1 = 0) {
    constexpr int RC = 2 * NC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = LT > 0 ? LT : pl.L;
    const int CS = col_stride(L);
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* buf = tw + L;
    double2* tmp = buf + NC * CS + RC;
    stage_twiddles<double2, NT>(tw, twd, L);
    const int b0 = bx * RC;
    const long long obase = (long long)by * so;
    for (int e = threadIdx.x; e < RC * len; e += NT) {
        const int li = e % RC, m = e / RC;
        const int b = b0 + li;
        double* slot = reinterpret_cast<double*>(&buf[(li >> 1) * CS + sk(m)]) + (li & 1);
        const bool inner = m >= 1 && m <= len - 2;
        double* mir = reinterpret_cast<double*>(&buf[(li >> 1) * CS + sk(inner ? L - m : m)]) + (li & 1);
        if (b < nb) {
            if constexpr (FROM_TMP) {
                const double v = igf_G_at(in, t0, t1, b, by, m);
                *slot = v;
                if (inner) *mir = v;
            } else {
                const double* src = in + (long long)b * sb + obase + (long long)m * se;
                cp_elem(slot, src);
                if (inner) cp_elem(mir, src);
            }
        } else {
            *slot = 0.0;
            if (inner) *mir = 0.0;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const double2* o = block_fft<double, false, LT, NC, NT>(buf, tmp, pl, tw);
    for (int e = threadIdx.x; e < RC * len; e += NT) {
        const int li = e % RC, m = e / RC;
        const int b = b0 + li;
        if (b >= nb) continue;
        const double2 v = o[(li >> 1) * CS + sk(m)];
        out[(long long)b * sb + obase + (long long)m * se] = (TO)((li & 1) ? v.y : v.x);
    }
}
template <typename TO, int LT, int NC, int NT, bool FROM_TMP = false>
__global__ void __launch_bounds__(NT, 1024 / NT) k_dct_lines(const double* __restrict__ in, TO* __restrict__ out, int len, int nb,
                                                  long long sb, long long so, long long se, FftPlan pl,
                                                  const double2* __restrict__ twd, int t0, int t1) {
    dct_lines_body<TO, LT, NC, NT, FROM_TMP>(in, out, len, nb, sb, so, se, pl, twd, blockIdx.x, blockIdx.y, t0, t1);
}

// The same cosine transforms for 256-point extensions with the
// register-resident line transform: two real lines per complex line (lines
// 2p and 2p + 1 as its real and imaginary parts, as in dct_lines_body), 8
// threads per complex line with the lanes along p, so one access reads
// consecutive lines; thread a holds the extension's elements a + 8m.  The
// butterflies, twiddles and operation order are block_fft's, so Ĝ has the
// same bits.
template <typename TO, int L>
__global__ void __launch_bounds__(LineGeo<L>::NT) k_dct_lines_reg(const double* __restrict__ in, TO* __restrict__ out,
                                                                 int len, int nb, long long sb, long long so,
                                                                 long long se, const double2* __restrict__ twd) {
    using C = Cx<double>;
    using G = LineGeo<L>;
    constexpr int M = G::M;
    __shared__ __align__(16) C xbuf[G::LINES][G::BUF + 1];
    const int li = threadIdx.x % G::LINES, a = threadIdx.x / G::LINES;
    const int p = blockIdx.x * G::LINES + li;
    const int b0 = 2 * p, b1 = 2 * p + 1;
    const long long obase = (long long)blockIdx.y * so;
    C v[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int e = a + 8 * m;
        const long long src = e <= L / 2 ? e : L - e;  // the even extension
        const double re = b0 < nb ? in[(long long)b0 * sb + obase + src * se] : 0.0;
        const double im = b1 < nb ? in[(long long)b1 * sb + obase + src * se] : 0.0;
        v[m] = C{re, im};
    }
    line_fft<double, false, false, L, true>(v, a, xbuf[li], reinterpret_cast<const C*>(twd));
    if (b0 >= nb) return;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int e = a + 8 * m;
        if (e < len) {
            out[(long long)b0 * sb + obase + (long long)e * se] = (TO)v[m].x;
            if (b1 < nb) out[(long long)b1 * sb + obase + (long long)e * se] = (TO)v[m].y;
        }
    }
}

// Full real transform of lines of length L along z (stride se), 2 NC lines
// per block packed two per complex FFT and split by the Hermitian symmetry,
// as pass A; the half spectrum k in [0, L/2] of line b goes to
// out[k * nb + b], negated with NEG (imgrho2tr = -rho2tr * grntr,
// FFTPoissonSolver.cpp:316).
template <typename TO, int LT, int NC, int NT, bool NEG = true>
__device__ __forceinline__ void rfft_lines_neg_body(const double* __restrict__ in, Cx<TO>* __restrict__ out, int nb,
                                                    long long se, const FftPlan& pl, const double2* __restrict__ twd,
                                                    int bx) {
    constexpr int RC = 2 * NC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = LT > 0 ? LT : pl.L;
    const int CS = col_stride(L);
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* buf = tw + L;
    double2* tmp = buf + NC * CS + RC;
    stage_twiddles<double2, NT>(tw, twd, L);
    const int b0 = bx * RC;
    for (int e = threadIdx.x; e < RC * L; e += NT) {
        const int li = e % RC, m = e / RC;
        const int b = b0 + li;
        double* slot = reinterpret_cast<double*>(&buf[(li >> 1) * CS + sk(m)]) + (li & 1);
        if (b < nb)
            cp_elem(slot, in + b + (long long)m * se);
        else
            *slot = 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    const double2* o = block_fft<double, false, LT, NC, NT>(buf, tmp, pl, tw);
    const int half = L / 2;
    for (int e = threadIdx.x; e < RC * (half + 1); e += NT) {
        const int li = e % RC, k = e / RC;
        const int b = b0 + li;
        if (b >= nb) continue;
        const int q = li >> 1;
        const double2 Z = o[q * CS + sk(k)];
        const double2 Zm = o[q * CS + sk(k == 0 ? 0 : L - k)];
        double re, im;
        if ((li & 1) == 0) {
            re = 0.5 * (Z.x + Zm.x);
            im = 0.5 * (Z.y - Zm.y);
        } else {
            re = 0.5 * (Z.y + Zm.y);
            im = -0.5 * (Z.x - Zm.x);
        }
        out[(long long)k * nb + b] = NEG ? Cx<TO>{(TO)(-re), (TO)(-im)} : Cx<TO>{(TO)re, (TO)im};
    }
}
template <typename TO, int LT, int NC, int NT, bool NEG = true>
__global__ void __launch_bounds__(NT, 1024 / NT) k_rfft_lines_neg(const double* __restrict__ in, Cx<TO>* __restrict__ out, int nb,
                                                       long long se, FftPlan pl, const double2* __restrict__ twd) {
    rfft_lines_neg_body<TO, LT, NC, NT, NEG>(in, out, nb, se, pl, twd, blockIdx.x);
}

// Tile-shape variants of a length: V = 0 is the widest shape (cols_for
// columns, up to 256 threads), each further variant halves the columns per
// block (more, smaller blocks, down to a single warp for the long
// transforms), which shortens each block's chain of barriers.  The batched
// autotuner picks per length; single-bunch launches use single_variant().
__host__ __device__ constexpr int cols_v(int LT, int V) {
    const int c = cols_for(LT) >> V;
    return c > 1 ? c : 1;
}
__host__ __device__ constexpr int threads_v(int LT, int V) {
    if (LT == 0) return 256;
    const int t = cols_v(LT, V) * (LT / min_radix(LT));
    return t < 32 ? 32 : t;
}

// ---------------------------------------------------------------- dispatch
template <int LT, int V = 0>
struct Geo {
    static constexpr int NC = cols_v(LT, V);
    static constexpr int NT = threads_v(LT, V);
};

// Tile-shape variant of single-bunch launches for a transform length (0 for
// lengths without a template instance): SCGPU_FFT_VARIANT=v forces one for
// every length, otherwise the measured default of the length.
int single_variant(int LT) {
    static const int forced = [] {
        const char* e = std::getenv("SCGPU_FFT_VARIANT");
        const int v = e ? std::atoi(e) : -1;
        return (v >= 0 && v < kFftLinesVariant) ? v : -1;
    }();
    if (LT == 0) return 0;
    if (forced >= 0) return forced;
    return LT >= 64 ? 1 : 0;  // half-width tiles measured faster from 64 points up (the cosine transforms most)
}

// Passes A (open z), B, C and D of 64-, 128- and 256-point lines take the
// register-resident kernels (k_*_lines, the same bits as the staged ones);
// pass E stays staged (its line form measured slower: 10.1 against 7.0 us
// at 128 points, 32.6 against 26.2 us at 256).  SCGPU_FFT_LINES=0 selects
// the staged kernels everywhere.
bool register_lines() {
    static const bool on = [] {
        const char* e = std::getenv("SCGPU_FFT_LINES");
        return !(e && std::string(e) == "0");
    }();
    return on;
}

// Calls f.template go<LT, V>() with V = single_variant(LT).
template <int LT, typename F>
void with_variant(F& f) {
    switch (single_variant(LT)) {
        case 1: f.template go<LT, 1>(); break;
        case 2: f.template go<LT, 2>(); break;
        case 3: f.template go<LT, 3>(); break;
        default: f.template go<LT, 0>(); break;
    }
}

template <typename C>
size_t smem_of(int L, int nc) {
    return sizeof(C) * tile_elems(L, nc);
}

template <typename TI>
size_t smem_conv(int L, int nc) {
    return (sizeof(double2) + sizeof(Cx<TI>)) * (size_t)L + 2 * sizeof(double2) * (size_t)nc * col_stride(L);
}

// Calls f.template run<LT>() with LT the template length for L, or 0.
template <typename F>
void with_length(int L, F&& f) {
    switch (L) {
        case 32: f.template run<32>(); break;
        case 64: f.template run<64>(); break;
        case 96: f.template run<96>(); break;
        case 128: f.template run<128>(); break;
        case 256: f.template run<256>(); break;
        default: f.template run<0>(); break;
    }
}

template <typename T, bool FULL = false>
struct LaunchA {
    const T* rho;
    Cx<T>* spec;
    int n0, n1, n2, L0, L1;
    FftPlan pz;
    const Cx<T>* twz;
    cudaStream_t s;
    template <int LT>
    void run() {
        if constexpr (!FULL && (LT == 64 || LT == 128 || LT == 256)) {
            if (register_lines() && 2 * n2 == LT) {
                using G = LineGeo<LT>;
                const long long lines = (long long)n1 * ((n0 + 1) / 2);
                k_fft_z_r2c_lines<T, LT><<<(unsigned)((lines + G::LINES - 1) / G::LINES), G::NT, 0, s>>>(
                    rho, spec, n0, n1, L0, L1, twz);
                return;
            }
        }
        with_variant<LT>(*this);
    }
    template <int LT, int V>
    void go() {
        constexpr int NC = Geo<LT, V>::NC, NT = Geo<LT, V>::NT;
        dim3 g((unsigned)((n0 + 2 * NC - 1) / (2 * NC)), (unsigned)n1);
        k_fft_z_r2c<T, LT, NC, NT, FULL><<<g, NT, smem_of<Cx<T>>(pz.L, NC), s>>>(rho, spec, n0, n1, n2, L0, L1, pz, twz);
    }
};

template <typename T, bool INV>
struct LaunchY {
    Cx<T>* spec;
    int n0, L0, n_in, n_out, planes;
    FftPlan py;
    const Cx<T>* twy;
    cudaStream_t s;
    template <int LT>
    void run() {
        if constexpr (LT == 64 || LT == 128 || LT == 256) {
            if (register_lines() && 2 * (INV ? n_out : n_in) == LT) {
                using G = LineGeo<LT>;
                const dim3 g((unsigned)((n0 + G::LINES - 1) / G::LINES), (unsigned)planes);
                k_fft_y_lines<T, INV, LT><<<g, G::NT, 0, s>>>(spec, n0, L0, planes, twy);
                return;
            }
        }
        with_variant<LT>(*this);
    }
    template <int LT, int V>
    void go() {
        constexpr int NC = Geo<LT, V>::NC, NT = Geo<LT, V>::NT;
        dim3 g((unsigned)((n0 + NC - 1) / NC), (unsigned)planes);
        k_fft_y<T, INV, LT, NC, NT><<<g, NT, smem_of<Cx<T>>(py.L, NC), s>>>(spec, n0, L0, n_in, n_out, py, twy);
    }
};

template <typename TI, bool CG = false>
struct LaunchC {
    const Cx<TI>* in;
    double2* out;
    const TI* ghat;
    int n0, n1, L1, rows;
    FftPlan px;
    const Cx<TI>* twi;
    const double2* two;
    cudaStream_t s;
    template <int LT>
    void run() {
        if constexpr (LT == 64 || LT == 128 || LT == 256) {
            if (register_lines() && 2 * n0 == LT) {
                using G = LineGeo<LT>;
                k_fft_x_conv_lines<TI, double, CG, LT><<<(unsigned)((rows + G::LINES - 1) / G::LINES), G::NT, 0, s>>>(
                    in, out, ghat, n0, n1, L1, rows, twi, two);
                return;
            }
        }
        with_variant<LT>(*this);
    }
    template <int LT, int V>
    void go() {
        constexpr int NC = Geo<LT, V>::NC, NT = Geo<LT, V>::NT;
        k_fft_x_conv<TI, double, LT, NC, NT, CG><<<(unsigned)((rows + NC - 1) / NC), NT, smem_conv<TI>(px.L, NC), s>>>(
            in, out, ghat, n0, n1, L1, rows, px, twi, two);
    }
};

template <typename TO, bool NEG = true>
struct LaunchRfftNeg {
    const double* in;
    Cx<TO>* out;
    int nb;
    long long se;
    FftPlan pl;
    const double2* tw;
    cudaStream_t s;
    template <int LT>
    void run() {
        with_variant<LT>(*this);
    }
    template <int LT, int V>
    void go() {
        constexpr int NC = Geo<LT, V>::NC, NT = Geo<LT, V>::NT;
        k_rfft_lines_neg<TO, LT, NC, NT, NEG>
            <<<(unsigned)((nb + 2 * NC - 1) / (2 * NC)), NT, smem_of<double2>(pl.L, NC), s>>>(in, out, nb, se, pl, tw);
    }
};

template <bool SELF, bool FLIP = false, bool FULL = false>
struct LaunchE {
    const double2* spec;
    double* phi;
    int n0, n1, n2, L0, L1;
    FftPlan pz;
    const double2* twz;
    const StepState* st;
    double normFact, coupling;
    cudaStream_t s;
    template <int LT>
    void run() {
        with_variant<LT>(*this);
    }
    template <int LT, int V>
    void go() {
        constexpr int NC = Geo<LT, V>::NC, NT = Geo<LT, V>::NT;
        dim3 g((unsigned)((n0 + 2 * NC - 1) / (2 * NC)), (unsigned)n1);
        k_fft_z_c2r<double, SELF, LT, NC, NT, FLIP, FULL><<<g, NT, smem_of<double2>(pz.L, NC), s>>>(
            spec, phi, n0, n1, n2, L0, L1, pz, twz, st, normFact, coupling);
    }
};

template <typename TO, bool FROM_TMP = false>
struct LaunchDct {
    const double* in;
    TO* out;
    int len, nb, outer;
    long long sb, so, se;
    FftPlan pl;
    const double2* tw;
    cudaStream_t s;
    int t0 = 0, t1 = 0;
    template <int LT>
    void run() {
        // 256-point lines only: at 128 points the staged tiles measured faster
        // (Green's-function phase 41.6 against 45.6 us at 64^3), at 256 points
        // the line form (185 against 175 us at 128^3)
        if constexpr (!FROM_TMP && LT == 256) {
            if (register_lines() && pl.L == LT && len == LT / 2 + 1) {
                using G = LineGeo<LT>;
                const int pairs = (nb + 1) / 2;
                dim3 g((unsigned)((pairs + G::LINES - 1) / G::LINES), (unsigned)outer);
                k_dct_lines_reg<TO, LT><<<g, G::NT, 0, s>>>(in, out, len, nb, sb, so, se, tw);
                return;
            }
        }
        with_variant<LT>(*this);
    }
    template <int LT, int V>
    void go() {
        constexpr int NC = Geo<LT, V>::NC, NT = Geo<LT, V>::NT;
        dim3 g((unsigned)((nb + 2 * NC - 1) / (2 * NC)), (unsigned)outer);
        k_dct_lines<TO, LT, NC, NT, FROM_TMP><<<g, NT, smem_of<double2>(pl.L, NC), s>>>(in, out, len, nb, sb, so, se, pl,
                                                                                     tw, t0, t1);
    }
};

// Raises the dynamic shared-memory limit of every instance of one length.
struct SetLimits {
    template <typename K>
    static void allow(K kernel) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    }
    template <int LT>
    void run() {
        go<LT, 0>();
        if constexpr (LT > 0) {
            go<LT, 1>();
            go<LT, 2>();
            go<LT, 3>();
        }
    }
    template <int LT, int V>
    void go() {
        constexpr int NC = Geo<LT, V>::NC, NT = Geo<LT, V>::NT;
        allow(k_fft_z_r2c<double, LT, NC, NT>);
        allow(k_fft_z_r2c<float, LT, NC, NT>);
        allow(k_fft_y<double, false, LT, NC, NT>);
        allow(k_fft_y<float, false, LT, NC, NT>);
        allow(k_fft_y<double, true, LT, NC, NT>);
        allow(k_fft_x_conv<double, double, LT, NC, NT>);
        allow(k_fft_x_conv<float, double, LT, NC, NT>);
        allow(k_fft_z_c2r<double, true, LT, NC, NT>);
        allow(k_fft_z_c2r<double, false, LT, NC, NT>);
        allow(k_dct_lines<double, LT, NC, NT>);
        allow(k_dct_lines<float, LT, NC, NT>);
        allow(k_dct_lines<double, LT, NC, NT, true>);
        allow(k_fft_x_conv<double, double, LT, NC, NT, true>);
        allow(k_fft_x_conv<float, double, LT, NC, NT, true>);
        allow(k_fft_z_c2r<double, true, LT, NC, NT, true>);
        allow(k_fft_z_c2r<double, false, LT, NC, NT, true>);
        allow(k_rfft_lines_neg<double, LT, NC, NT>);
        allow(k_rfft_lines_neg<float, LT, NC, NT>);
        allow(k_rfft_lines_neg<double, LT, NC, NT, false>);
        allow(k_rfft_lines_neg<float, LT, NC, NT, false>);
        allow(k_fft_z_r2c<double, LT, NC, NT, true>);
        allow(k_fft_z_r2c<float, LT, NC, NT, true>);
        allow(k_fft_z_c2r<double, true, LT, NC, NT, false, true>);
        allow(k_fft_z_c2r<double, false, LT, NC, NT, false, true>);
    }
};

// ---------------------------------------------------------------- batches
__device__ __forceinline__ FftPlan plan_dev(int L) {
    const RadixPlan r = radix_plan(L);
    FftPlan p;
    p.L = L;
    p.nst = r.nst;
#pragma unroll
    for (int i = 0; i < 12; ++i) p.r[i] = r.r[i];
    return p;
}

// twiddles of axis a as complex T (the float table follows the double one)
template <typename T>
__device__ __forceinline__ const Cx<T>* tw_dev(const DevBunch& d, int a) {
    const double2* p = reinterpret_cast<const double2*>(d.tw[a]);
    if constexpr (sizeof(T) == sizeof(double))
        return reinterpret_cast<const Cx<T>*>(p);
    else
        return reinterpret_cast<const Cx<T>*>(p + 2 * d.bc.n[a]);
}

// One kernel per pass: block i runs the single-bunch body for bunch work[i].x
// at block coordinates (work[i].y, work[i].z), with that bunch's sizes and
// buffers (T: the forward-half type, as in convolution_t).
template <typename T, int PASS, int LT, int NC, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_fft_pass_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work,
                                                        int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    const int n0 = d.bc.n[0], n1 = d.bc.n[1], n2 = d.bc.n[2];
    const int L0 = 2 * n0, L1 = 2 * n1, L2 = 2 * n2;
    Cx<T>* fwd = reinterpret_cast<Cx<T>*>(d.precision == 0 ? d.spec : d.spec_lo);
    double2* inv = reinterpret_cast<double2*>(d.spec);
    if constexpr (PASS == kPassZR2C) {
        fft_z_r2c_body<T, LT, NC, NT>((const T*)d.rho, fwd, n0, n1, n2, L0, L1, plan_dev(L2), tw_dev<T>(d, 2), w.y, w.z);
    } else if constexpr (PASS == kPassYFwd) {
        fft_y_body<T, false, LT, NC, NT>(fwd, n0, L0, n1, L1, plan_dev(L1), tw_dev<T>(d, 1), w.y, w.z);
    } else if constexpr (PASS == kPassXConv) {
        fft_x_conv_body<T, double, LT, NC, NT>(fwd, inv, (const T*)d.ghat, n0, n1, L1, (n2 + 1) * L1, plan_dev(L0),
                                               tw_dev<T>(d, 0), tw_dev<double>(d, 0), w.y);
    } else if constexpr (PASS == kPassYInv) {
        fft_y_body<double, true, LT, NC, NT>(inv, n0, L0, L1, n1, plan_dev(L1), tw_dev<double>(d, 1), w.y, w.z);
    } else if constexpr (PASS == kPassZC2R) {
        double normFact = 1.0;
        normFact /= L0;
        normFact /= L1;
        normFact /= L2;
        fft_z_c2r_body<double, true, LT, NC, NT>(inv, d.phi, n0, n1, n2, L0, L1, plan_dev(L2), tw_dev<double>(d, 2), d.st,
                                                 normFact, d.bc.coupling, w.y, w.z);
    } else {
        const long long g0 = n0 + 1, g1 = n1 + 1, g2 = n2 + 1;
        // G formed from the antiderivative in the z pass (gtmp -> gline ->
        // gtmp -> ghat), as launch_green_transform_from_tmp
        if constexpr (PASS == kPassDctZ)
            dct_lines_body<double, LT, NC, NT, true>(d.gtmp, d.gline, (int)g2, (int)g0, 1, g0, g0 * g1, plan_dev(L2),
                                                     tw_dev<double>(d, 2), w.y, w.z, n0 + 2, n1 + 2);
        else if constexpr (PASS == kPassDctY)
            dct_lines_body<double, LT, NC, NT>(d.gline, d.gtmp, (int)g1, (int)g0, 1, g0 * g1, g0, plan_dev(L1),
                                               tw_dev<double>(d, 1), w.y, w.z);
        else
            dct_lines_body<T, LT, NC, NT>(d.gtmp, (T*)d.ghat, (int)g0, (int)g1, g0, g0 * g1, 1, plan_dev(L0),
                                          tw_dev<double>(d, 0), w.y, w.z);
    }
}

inline bool line_length(int L) { return L == 64 || L == 128 || L == 256; }

// Variant kFftLinesVariant: passes B, C and D of 64-, 128- and 256-point
// lines run the register-resident line transforms (the same bits), block
// (x, y) of a bunch as in the single-bunch launch.
template <typename T, int PASS, int L>
__global__ void __launch_bounds__(LineGeo<L>::NT) k_fft_lines_batch(const DevBunch* __restrict__ tab,
                                                                  const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    const int n0 = d.bc.n[0], n1 = d.bc.n[1], n2 = d.bc.n[2];
    const int L0 = 2 * n0, L1 = 2 * n1;
    Cx<T>* fwd = reinterpret_cast<Cx<T>*>(d.precision == 0 ? d.spec : d.spec_lo);
    double2* inv = reinterpret_cast<double2*>(d.spec);
    if constexpr (PASS == kPassYFwd)
        fft_y_lines_body<T, false, L>(fwd, n0, L0, n2 + 1, tw_dev<T>(d, 1), w.y, w.z);
    else if constexpr (PASS == kPassXConv)
        fft_x_conv_lines_body<T, double, false, L>(fwd, inv, (const T*)d.ghat, n0, n1, L1, (n2 + 1) * L1, tw_dev<T>(d, 0),
                                                   tw_dev<double>(d, 0), w.y);
    else
        fft_y_lines_body<double, true, L>(inv, n0, L0, n2 + 1, tw_dev<double>(d, 1), w.y, w.z);
}

template <typename T, int PASS>
struct LaunchLinesBatch {
    const DevBunch* tab;
    const int4* work;
    int nitems, n;
    cudaStream_t s;
    template <int LT>
    void run() {
        if constexpr (LT == 64 || LT == 128 || LT == 256)
            k_fft_lines_batch<T, PASS, LT><<<n, LineGeo<LT>::NT, 0, s>>>(tab, work, nitems);
    }
};

template <typename T, int PASS>
size_t pass_smem(int L, int nc) {
    if constexpr (PASS == kPassXConv) return smem_conv<T>(L, nc);
    if constexpr (PASS == kPassZR2C || PASS == kPassYFwd) return smem_of<Cx<T>>(L, nc);
    return smem_of<double2>(L, nc);
}

template <typename T, int PASS, int V>
struct LaunchPassBatch {
    const DevBunch* tab;
    const int4* work;
    int nitems, n, L;
    cudaStream_t s;
    template <int LT>
    void run() {
        constexpr int NC = cols_v(LT, V), NT = threads_v(LT, V);
        auto k = k_fft_pass_batch<T, PASS, LT, NC, NT>;
        const size_t sm = pass_smem<T, PASS>(L, NC);
        static bool limits = [&] {
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
            return true;
        }();
        (void)limits;
        k<<<n, NT, sm, s>>>(tab, work, nitems);
    }
};

template <typename T, int PASS>
void pass_batch_t(int L, int variant, const DevBunch* tab, const int4* work, int nitems, int n, cudaStream_t s) {
    if (variant == kFftLinesVariant) {
        if constexpr (PASS == kPassYFwd || PASS == kPassXConv || PASS == kPassYInv) {
            if (line_length(L)) {
                with_length(L, LaunchLinesBatch<T, PASS>{tab, work, nitems, n, s});
                return;
            }
        }
        variant = 0;  // the other passes with the widest tiles
    }
    switch (variant) {
        case 1: with_length(L, LaunchPassBatch<T, PASS, 1>{tab, work, nitems, n, L, s}); break;
        case 2: with_length(L, LaunchPassBatch<T, PASS, 2>{tab, work, nitems, n, L, s}); break;
        case 3: with_length(L, LaunchPassBatch<T, PASS, 3>{tab, work, nitems, n, L, s}); break;
        default: with_length(L, LaunchPassBatch<T, PASS, 0>{tab, work, nitems, n, L, s}); break;
    }
}

template <typename T>
void pass_batch(int pass, int L, int variant, const DevBunch* tab, const int4* work, int nitems, int n, cudaStream_t s) {
    switch (pass) {
        case kPassZR2C: pass_batch_t<T, kPassZR2C>(L, variant, tab, work, nitems, n, s); break;
        case kPassYFwd: pass_batch_t<T, kPassYFwd>(L, variant, tab, work, nitems, n, s); break;
        case kPassXConv: pass_batch_t<T, kPassXConv>(L, variant, tab, work, nitems, n, s); break;
        case kPassYInv: pass_batch_t<T, kPassYInv>(L, variant, tab, work, nitems, n, s); break;
        case kPassZC2R: pass_batch_t<T, kPassZC2R>(L, variant, tab, work, nitems, n, s); break;
        case kPassDctZ: pass_batch_t<T, kPassDctZ>(L, variant, tab, work, nitems, n, s); break;
        case kPassDctY: pass_batch_t<T, kPassDctY>(L, variant, tab, work, nitems, n, s); break;
        default: pass_batch_t<T, kPassDctX>(L, variant, tab, work, nitems, n, s); break;
    }
}

inline bool special_length(int L) { return L == 32 || L == 64 || L == 96 || L == 128 || L == 256; }

}  // namespace

bool fft_register_lines() { return register_lines(); }

int fft_pass_length(int pass, const DevBunch& b) {
    switch (pass) {
        case kPassZR2C:
        case kPassZC2R:
        case kPassDctZ: return 2 * b.bc.n[2];
        case kPassYFwd:
        case kPassYInv:
        case kPassDctY: return 2 * b.bc.n[1];
        default: return 2 * b.bc.n[0];
    }
}

void fft_pass_grid(int pass, const DevBunch& b, int variant, int* gx, int* gy) {
    const int L = fft_pass_length(pass, b);
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    if (variant == kFftLinesVariant) {
        const int lines = L >= 256 ? LineGeo<256>::LINES : LineGeo<128>::LINES;
        if (line_length(L) && (pass == kPassYFwd || pass == kPassYInv)) {
            *gx = (n0 + lines - 1) / lines;
            *gy = n2 + 1;
            return;
        }
        if (line_length(L) && pass == kPassXConv) {
            *gx = ((n2 + 1) * 2 * n1 + lines - 1) / lines;
            *gy = 1;
            return;
        }
        variant = 0;
    }
    const int nc = cols_v(special_length(L) ? L : 0, variant);
    switch (pass) {
        case kPassZR2C:
        case kPassZC2R:
            *gx = (n0 + 2 * nc - 1) / (2 * nc);
            *gy = n1;
            break;
        case kPassYFwd:
        case kPassYInv:
            *gx = (n0 + nc - 1) / nc;
            *gy = n2 + 1;
            break;
        case kPassXConv:
            *gx = ((n2 + 1) * 2 * n1 + nc - 1) / nc;
            *gy = 1;
            break;
        case kPassDctZ:
            *gx = (n0 + 1 + 2 * nc - 1) / (2 * nc);
            *gy = n1 + 1;
            break;
        case kPassDctY:
            *gx = (n0 + 1 + 2 * nc - 1) / (2 * nc);
            *gy = n2 + 1;
            break;
        default:
            *gx = (n1 + 1 + 2 * nc - 1) / (2 * nc);
            *gy = n2 + 1;
            break;
    }
}

void launch_fft_pass_batch(int pass, int L, int precision, int variant, const DevBunch* tab, const int4* work, int nitems,
                           int n, cudaStream_t s) {
    if (n <= 0 || nitems <= 0) return;
    if (precision == 0)
        pass_batch<double>(pass, L, variant, tab, work, nitems, n, s);
    else
        pass_batch<float>(pass, L, variant, tab, work, nitems, n, s);
}

FftPlan make_plan(int L) {
    const RadixPlan r = radix_plan(L);
    FftPlan p{};
    p.L = L;
    p.nst = r.nst;
    for (int i = 0; i < 12; ++i) p.r[i] = r.r[i];
    return p;
}

size_t fft_smem_bytes(const DevBunch& b) {
    size_t m = 0;
    for (int d = 0; d < 3; ++d) {
        const int L = 2 * b.bc.n[d];
        m = std::max(m, smem_of<double2>(L, cols_for(0)));
        m = std::max(m, smem_conv<double>(L, cols_for(0)));
    }
    return m;
}

// Axis d's transform length: the doubled grid, except z with periodic z.
static inline int axis_length(const DevBunch& b, int d) {
    return (d == 2 && b.periodic_z) ? b.bc.n[2] : 2 * b.bc.n[d];
}

// twiddles exp(-2 pi i e / L), e in [0, L), from long double arithmetic
// rounded once to the table's type (tf may be null)
void twiddle_values(int L, double2* td, float2* tf) {
    for (int e = 0; e < L; ++e) {
        const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)e / (long double)L;
        td[e] = double2{(double)cosl(a), (double)sinl(a)};
        if (tf) tf[e] = float2{(float)cosl(a), (float)sinl(a)};
    }
}

void upload_twiddles(DevBunch& b, cudaStream_t s) {
    for (int d = 0; d < 3; ++d) {
        const int L = axis_length(b, d);
        std::vector<double2> td(L);
        std::vector<float2> tf(L);
        twiddle_values(L, td.data(), tf.data());
        // the double table always (the G spectrum is built in FP64); the float one in the mixed form
        double2* dptr = reinterpret_cast<double2*>(b.tw[d]);
        cudaMemcpyAsync(dptr, td.data(), L * sizeof(double2), cudaMemcpyHostToDevice, s);
        if (b.precision != 0) {
            float2* fptr = reinterpret_cast<float2*>(dptr + L);
            cudaMemcpyAsync(fptr, tf.data(), L * sizeof(float2), cudaMemcpyHostToDevice, s);
        }
    }
    cudaStreamSynchronize(s);
}

static inline const void* tw_for(const DevBunch& b, int d) {
    const int L = axis_length(b, d);
    const double2* dptr = reinterpret_cast<const double2*>(b.tw[d]);
    return b.precision == 0 ? (const void*)dptr : (const void*)(dptr + L);
}

// Spectrum of the mirrored G from b.gline ((n0+1)(n1+1)(n2+1), FP64), into b.ghat.
void launch_green_transform(const DevBunch& b, cudaStream_t s) {
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long g0 = n0 + 1, g1 = n1 + 1, g2 = n2 + 1;
    const FftPlan p0 = make_plan(2 * n0), p1 = make_plan(2 * n1), p2 = make_plan(2 * n2);
    const double2* tw0 = reinterpret_cast<const double2*>(b.tw[0]);
    const double2* tw1 = reinterpret_cast<const double2*>(b.tw[1]);
    const double2* tw2 = reinterpret_cast<const double2*>(b.tw[2]);
    // z lines: batch x (stride 1), outer y
    with_length(2 * n2, LaunchDct<double>{b.gline, b.gtmp, (int)g2, (int)g0, (int)g1, 1, g0, g0 * g1, p2, tw2, s});
    // y lines: batch x, outer z
    with_length(2 * n1, LaunchDct<double>{b.gtmp, b.gline, (int)g1, (int)g0, (int)g2, 1, g0 * g1, g0, p1, tw1, s});
    // x lines: batch y (stride g0), outer z
    if (b.precision == 0)
        with_length(2 * n0, LaunchDct<double>{b.gline, (double*)b.ghat, (int)g0, (int)g1, (int)g2, g0, g0 * g1, 1, p0, tw0, s});
    else
        with_length(2 * n0, LaunchDct<float>{b.gline, (float*)b.ghat, (int)g0, (int)g1, (int)g2, g0, g0 * g1, 1, p0, tw0, s});
}

// The same spectrum from the antiderivative (b.gtmp, launch_igf_tmp): the
// z transforms form G as they stage it and write gline, the y transforms
// gline -> gtmp, the x transforms gtmp -> ghat.  G's values and every
// transform are those of launch_igf + launch_green_transform, so Ĝ has the
// same bits; G is never stored.
void launch_green_transform_from_tmp(const DevBunch& b, cudaStream_t s) {
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long g0 = n0 + 1, g1 = n1 + 1, g2 = n2 + 1;
    const FftPlan p0 = make_plan(2 * n0), p1 = make_plan(2 * n1), p2 = make_plan(2 * n2);
    const double2* tw0 = reinterpret_cast<const double2*>(b.tw[0]);
    const double2* tw1 = reinterpret_cast<const double2*>(b.tw[1]);
    const double2* tw2 = reinterpret_cast<const double2*>(b.tw[2]);
    LaunchDct<double, true> z{b.gtmp, b.gline, (int)g2, (int)g0, (int)g1, 1, g0, g0 * g1, p2, tw2, s};
    z.t0 = n0 + 2;
    z.t1 = n1 + 2;
    with_length(2 * n2, z);
    with_length(2 * n1, LaunchDct<double>{b.gline, b.gtmp, (int)g1, (int)g0, (int)g2, 1, g0 * g1, g0, p1, tw1, s});
    if (b.precision == 0)
        with_length(2 * n0, LaunchDct<double>{b.gtmp, (double*)b.ghat, (int)g0, (int)g1, (int)g2, g0, g0 * g1, 1, p0, tw0, s});
    else
        with_length(2 * n0, LaunchDct<float>{b.gtmp, (float*)b.ghat, (int)g0, (int)g1, (int)g2, g0, g0 * g1, 1, p0, tw0, s});
}

// Spectrum of the image's shifted G (b.gimg, (n0+1)(n1+1)(2 n2), FP64):
// cosine transforms along y and x on every z plane (G is even in x and y),
// then a full real transform along z (it is not even in z), negated, into
// b.ghat_img (n2+1)(n1+1)(n0+1) complex T.
void launch_green_transform_image(const DevBunch& b, cudaStream_t s) {
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long g0 = n0 + 1, g1 = n1 + 1, L2 = 2 * n2;
    const long long GI = g0 * g1 * L2;
    const FftPlan p0 = make_plan(2 * n0), p1 = make_plan(2 * n1), p2 = make_plan(2 * n2);
    const double2* tw0 = reinterpret_cast<const double2*>(b.tw[0]);
    const double2* tw1 = reinterpret_cast<const double2*>(b.tw[1]);
    const double2* tw2 = reinterpret_cast<const double2*>(b.tw[2]);
    double* ga = b.gimg;
    double* gb = b.gimg + GI;
    // y lines: batch x, outer z (2 n2 planes)
    with_length(2 * n1, LaunchDct<double>{ga, gb, (int)g1, (int)g0, (int)L2, 1, g0 * g1, g0, p1, tw1, s});
    // x lines: batch y (stride g0), outer z
    with_length(2 * n0, LaunchDct<double>{gb, ga, (int)g0, (int)g1, (int)L2, g0, g0 * g1, 1, p0, tw0, s});
    // z lines of length 2 n2: batch (x, y), element stride g0 g1
    if (b.precision == 0)
        with_length(2 * n2, LaunchRfftNeg<double>{ga, (double2*)b.ghat_img, (int)(g0 * g1), g0 * g1, p2, tw2, s});
    else
        with_length(2 * n2, LaunchRfftNeg<float>{ga, (float2*)b.ghat_img, (int)(g0 * g1), g0 * g1, p2, tw2, s});
}

// Periodic z (FFTPoissonSolver with bcz, :130-155, :661-662): G on its first
// n2 z planes (the unshifted G of b.gline, not mirrored in z), cosine
// transforms along y and x, then a full real transform of length n2 along z
// into b.ghat_img (complex T).
void launch_green_transform_periodic(const DevBunch& b, cudaStream_t s) {
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long g0 = n0 + 1, g1 = n1 + 1;
    const FftPlan p0 = make_plan(2 * n0), p1 = make_plan(2 * n1), pz = make_plan(n2);
    const double2* tw0 = reinterpret_cast<const double2*>(b.tw[0]);
    const double2* tw1 = reinterpret_cast<const double2*>(b.tw[1]);
    const double2* tw2 = reinterpret_cast<const double2*>(b.tw[2]);
    with_length(2 * n1, LaunchDct<double>{b.gline, b.gtmp, (int)g1, (int)g0, n2, 1, g0 * g1, g0, p1, tw1, s});
    with_length(2 * n0, LaunchDct<double>{b.gtmp, b.gline, (int)g0, (int)g1, n2, g0, g0 * g1, 1, p0, tw0, s});
    if (b.precision == 0)
        with_length(n2, LaunchRfftNeg<double, false>{b.gline, (double2*)b.ghat_img, (int)(g0 * g1), g0 * g1, pz, tw2, s});
    else
        with_length(n2, LaunchRfftNeg<float, false>{b.gline, (float2*)b.ghat_img, (int)(g0 * g1), g0 * g1, pz, tw2, s});
}

// T is the type of the forward half (A, B and the forward x transform of C);
// the inverse half (C's inverse, D, E) is FP64 in both forms.  With energy
// bins the plain form keeps the forward spectrum in b.spec_fwd, so the bin's
// own and its image's convolutions (C, D, E twice) start from one A, B.
// parts: kConvForwardPart (A, B: need only rho) and/or kConvRestPart (C, D,
// E: need the spectrum of G as well).
template <typename T>
static void convolution_t(const DevBunch& b, int mode, int parts, cudaStream_t s) {
    using C = Cx<T>;
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const int L0 = 2 * n0, L1 = 2 * n1, L2 = axis_length(b, 2);
    const int K = L2 / 2;  // half-spectrum planes 0..K along z
    const FftPlan px = make_plan(L0), py = make_plan(L1), pz = make_plan(L2);
    const C* twx = reinterpret_cast<const C*>(tw_for(b, 0));
    const C* twy = reinterpret_cast<const C*>(tw_for(b, 1));
    const C* twz = reinterpret_cast<const C*>(tw_for(b, 2));
    const double2* twx_d = reinterpret_cast<const double2*>(b.tw[0]);
    const double2* twy_d = reinterpret_cast<const double2*>(b.tw[1]);
    const double2* twz_d = reinterpret_cast<const double2*>(b.tw[2]);
    C* fwd = reinterpret_cast<C*>(b.precision == 0 ? (b.spec_fwd ? b.spec_fwd : b.spec) : b.spec_lo);
    double2* inv = reinterpret_cast<double2*>(b.spec);
    double normFact = 1.0;
    normFact /= L0;
    normFact /= L1;
    normFact /= L2;
    if (parts & kConvForwardPart) {
        if (b.periodic_z)
            with_length(L2, LaunchA<T, true>{(const T*)b.rho, fwd, n0, n1, n2, L0, L1, pz, twz, s});
        else
            with_length(L2, LaunchA<T>{(const T*)b.rho, fwd, n0, n1, n2, L0, L1, pz, twz, s});
        with_length(L1, LaunchY<T, false>{fwd, n0, L0, n1, L1, K + 1, py, twy, s});
    }
    if ((parts & kConvRestPart) && b.periodic_z) {
        with_length(L0, LaunchC<T, true>{fwd, inv, (const T*)b.ghat_img, n0, n1, L1, (K + 1) * L1, px, twx, twx_d, s});
        with_length(L1, LaunchY<double, true>{inv, n0, L0, L1, n1, K + 1, py, twy_d, s});
        if (mode == kConvSelfField)
            with_length(L2, LaunchE<true, false, true>{inv, b.phi, n0, n1, n2, L0, L1, pz, twz_d, b.st, normFact,
                                                       b.bc.coupling, s});
        else
            with_length(L2, LaunchE<false, false, true>{inv, b.phi, n0, n1, n2, L0, L1, pz, twz_d, b.st, normFact,
                                                        b.bc.coupling, s});
        return;
    }
    if (parts & kConvRestPart) {
        with_length(L0, LaunchC<T>{fwd, inv, (const T*)b.ghat, n0, n1, L1, (n2 + 1) * L1, px, twx, twx_d, s});
        with_length(L1, LaunchY<double, true>{inv, n0, L0, L1, n1, n2 + 1, py, twy_d, s});
        if (mode == kConvSelfField)
            with_length(L2, LaunchE<true>{inv, b.phi, n0, n1, n2, L0, L1, pz, twz_d, b.st, normFact, b.bc.coupling, s});
        else
            with_length(L2, LaunchE<false>{inv, b.phi, n0, n1, n2, L0, L1, pz, twz_d, b.st, normFact, b.bc.coupling, s});
    }
    if (parts & kConvImagePart) {
        with_length(L0, LaunchC<T, true>{fwd, inv, (const T*)b.ghat_img, n0, n1, L1, (n2 + 1) * L1, px, twx, twx_d, s});
        with_length(L1, LaunchY<double, true>{inv, n0, L0, L1, n1, n2 + 1, py, twy_d, s});
        if (mode == kConvSelfField)
            with_length(L2, LaunchE<true, true>{inv, b.phi, n0, n1, n2, L0, L1, pz, twz_d, b.st, normFact, b.bc.coupling, s});
        else
            with_length(L2,
                        LaunchE<false, true>{inv, b.phi, n0, n1, n2, L0, L1, pz, twz_d, b.st, normFact, b.bc.coupling, s});
    }
}

void launch_convolution(const DevBunch& b, int mode, cudaStream_t s) {
    launch_convolution_part(b, mode, kConvForwardPart | kConvRestPart, s);
}

void launch_convolution_part(const DevBunch& b, int mode, int parts, cudaStream_t s) {
    if (b.precision == 0)
        convolution_t<double>(b, mode, parts, s);
    else
        convolution_t<float>(b, mode, parts, s);
}

void fft_set_smem_limits() {
    SetLimits sl;
    sl.run<32>();
    sl.run<64>();
    sl.run<96>();
    sl.run<128>();
    sl.run<256>();
    sl.run<0>();
}

}  // namespace sc
