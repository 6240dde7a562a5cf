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
#include <cmath>
#include <vector>

#include "sc_internal.h"

namespace sc {
namespace {

constexpr int kThreads = 256;

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
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

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
    } else if constexpr (R == 16) {
        // 4 x 4: y_q = DFT4 over p of x_{q + 4p}; y_q[s] *= W16^{q s}; X_{s + 4t} = DFT4 over q of y_q[s]
        C y[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            C t[4] = {v[q], v[q + 4], v[q + 8], v[q + 12]};
            dft<T, 4, INV>(t);
#pragma unroll
            for (int s = 0; s < 4; ++s) y[q][s] = t[s];
        }
        const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173;  // cos, sin of 2 pi / 16
        const T c2 = (T)0.70710678118654752440;
        // W16^j = cos(2 pi j/16) - i sin(2 pi j/16) (forward), j = q s in {1, 2, 3, 4, 6, 9}
        const C w[10] = {C{(T)1, (T)0},  C{c1, -s1},       C{c2, -c2},      C{s1, -c1},  C{(T)0, (T)-1},
                         C{-s1, -c1},    C{-c2, -c2},      C{-c1, -s1},     C{(T)-1, (T)0}, C{-c1, s1}};
#pragma unroll
        for (int q = 1; q < 4; ++q)
#pragma unroll
            for (int s = 1; s < 4; ++s) {
                C tw = w[q * s];
                if (INV) tw.y = -tw.y;
                y[q][s] = cmul(y[q][s], tw);
            }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            C t[4] = {y[0][s], y[1][s], y[2][s], y[3][s]};
            dft<T, 4, INV>(t);
#pragma unroll
            for (int tt = 0; tt < 4; ++tt) v[s + 4 * tt] = t[tt];
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

// One Stockham autosort stage (radix R) over ncols columns of length L.
template <typename T, int R, bool INV>
__device__ __forceinline__ void stage(const Cx<T>* __restrict__ in, Cx<T>* __restrict__ out, int L, int Ns, int ncols,
                                      const Cx<T>* __restrict__ tw) {
    using C = Cx<T>;
    const int nb = L / R;
    const int step = L / (Ns * R);
    for (int w = threadIdx.x; w < ncols * nb; w += blockDim.x) {
        const int col = w / nb;
        const int j = w - col * nb;
        const C* src = in + col * L;
        C* dst = out + col * L;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[j + r * nb];
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; ++r) {
            C t = tw[r * k * step];
            if (INV) t.y = -t.y;
            v[r] = cmul(v[r], t);
        }
        dft<T, R, INV>(v);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
    }
}

// Complex FFT of ncols columns (buf[col * L + i]); result returned (buf or tmp).
template <typename T, bool INV>
__device__ Cx<T>* block_fft(Cx<T>* buf, Cx<T>* tmp, int ncols, const FftPlan& pl, const Cx<T>* tw) {
    int Ns = 1;
    Cx<T>* a = buf;
    Cx<T>* b = tmp;
    for (int s = 0; s < pl.nst; ++s) {
        const int R = pl.r[s];
        if (R == 16)
            stage<T, 16, INV>(a, b, pl.L, Ns, ncols, tw);
        else if (R == 8)
            stage<T, 8, INV>(a, b, pl.L, Ns, ncols, tw);
        else if (R == 4)
            stage<T, 4, INV>(a, b, pl.L, Ns, ncols, tw);
        else if (R == 2)
            stage<T, 2, INV>(a, b, pl.L, Ns, ncols, tw);
        else if (R == 3)
            stage<T, 3, INV>(a, b, pl.L, Ns, ncols, tw);
        else
            stage<T, 5, INV>(a, b, pl.L, Ns, ncols, tw);
        __syncthreads();
        Cx<T>* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

template <typename T>
__device__ __forceinline__ void load_twiddles(Cx<T>* dst, const Cx<T>* __restrict__ src, int L) {
    for (int e = threadIdx.x; e < L; e += blockDim.x) dst[e] = src[e];
}

// ---------------------------------------------------------------- pass A
template <typename T>
__global__ void __launch_bounds__(kThreads) k_fft_z_r2c(const T* __restrict__ rho, Cx<T>* __restrict__ spec, int n0, int n1,
                                                        int n2, int L0, int L1, FftPlan pz, const Cx<T>* __restrict__ twz) {
    using C = Cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L2 = pz.L;
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + L2;
    C* tmp = buf + 16 * L2 + 32;
    load_twiddles<T>(tw, twz, L2);
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * 32;
    for (int e = threadIdx.x; e < 32 * L2; e += blockDim.x) {
        const int xi = e & 31, z = e >> 5;
        const int x = x0 + xi;
        T v = (T)0;
        if (z < n2 && x < n0) v = rho[((size_t)z * n1 + y) * n0 + x];
        T* slot = reinterpret_cast<T*>(&buf[(xi >> 1) * L2 + z]);
        slot[xi & 1] = v;
    }
    __syncthreads();
    const C* out = block_fft<T, false>(buf, tmp, 16, pz, tw);
    for (int e = threadIdx.x; e < 32 * (n2 + 1); e += blockDim.x) {
        const int xi = e & 31, k = e >> 5;
        const int x = x0 + xi;
        if (x >= n0) continue;
        const int q = xi >> 1;
        const C Z = out[q * L2 + k];
        const C Zm = out[q * L2 + ((L2 - k) % L2)];
        C r;
        if ((xi & 1) == 0)
            r = C{(T)0.5 * (Z.x + Zm.x), (T)0.5 * (Z.y - Zm.y)};
        else
            r = C{(T)0.5 * (Z.y + Zm.y), (T)-0.5 * (Z.x - Zm.x)};
        spec[((size_t)k * L1 + y) * L0 + x] = r;
    }
}

// ---------------------------------------------------------------- pass B / D
template <typename T, bool INV>
__global__ void __launch_bounds__(kThreads) k_fft_y(Cx<T>* __restrict__ spec, int n0, int L0, int n_in, int n_out, FftPlan py,
                                                    const Cx<T>* __restrict__ twy) {
    using C = Cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L1 = py.L;
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + L1;
    C* tmp = buf + 16 * L1;
    load_twiddles<T>(tw, twy, L1);
    const int kz = blockIdx.y;
    const int x0 = blockIdx.x * 16;
    C* plane = spec + (size_t)kz * L1 * L0;
    for (int e = threadIdx.x; e < 16 * L1; e += blockDim.x) {
        const int xi = e & 15, yy = e >> 4;
        const int x = x0 + xi;
        C v = C{(T)0, (T)0};
        if (yy < n_in && x < n0) v = plane[(size_t)yy * L0 + x];
        buf[xi * L1 + yy] = v;
    }
    __syncthreads();
    const C* out = block_fft<T, INV>(buf, tmp, 16, py, tw);
    for (int e = threadIdx.x; e < 16 * n_out; e += blockDim.x) {
        const int xi = e & 15, yy = e >> 4;
        const int x = x0 + xi;
        if (x < n0) plane[(size_t)yy * L0 + x] = out[xi * L1 + yy];
    }
}

// ---------------------------------------------------------------- pass C
// The forward transform and the multiplication run in TI, the inverse in TO.
// The mixed form takes TI = float, TO = double: rounding in the forward half
// is white noise in the spectrum, which the derivative of phi does not
// amplify, while rounding after the multiplication would be noise relative
// to phi itself and is kept at FP64.  `in` and `out` alias in the plain form;
// every block reads its rows before it writes them.
constexpr int kRowsC = 8;
template <typename TI, typename TO>
__global__ void __launch_bounds__(kThreads) k_fft_x_conv(const Cx<TI>* in, Cx<TO>* out, const TI* __restrict__ ghat, int n0,
                                                         int n1, int L1, long long rows, FftPlan px,
                                                         const Cx<TI>* __restrict__ twi, const Cx<TO>* __restrict__ two) {
    using CI = Cx<TI>;
    using CO = Cx<TO>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L0 = px.L;
    CO* tw_o = reinterpret_cast<CO*>(smem_raw);
    CI* tw_i = reinterpret_cast<CI*>(tw_o + L0);
    CO* bufo = reinterpret_cast<CO*>(tw_i + L0);
    CO* tmpo = bufo + kRowsC * L0;
    load_twiddles<TO>(tw_o, two, L0);
    load_twiddles<TI>(tw_i, twi, L0);
    CI* bufi = reinterpret_cast<CI*>(bufo);
    CI* tmpi = reinterpret_cast<CI*>(tmpo);
    const long long r0 = (long long)blockIdx.x * kRowsC;
    for (int e = threadIdx.x; e < kRowsC * L0; e += blockDim.x) {
        const int ri = e / L0, x = e - ri * L0;
        const long long r = r0 + ri;
        CI v = CI{(TI)0, (TI)0};
        if (r < rows && x < n0) v = in[(size_t)r * L0 + x];
        bufi[ri * L0 + x] = v;
    }
    __syncthreads();
    const CI* f = block_fft<TI, false>(bufi, tmpi, kRowsC, px, tw_i);
    CO* g = (f == bufi) ? tmpo : bufo;
    CO* h = (f == bufi) ? bufo : tmpo;
    for (int e = threadIdx.x; e < kRowsC * L0; e += blockDim.x) {
        const int ri = e / L0, kx = e - ri * L0;
        const long long r = r0 + ri;
        if (r >= rows) continue;
        const int kz = (int)(r / L1);
        const int ky = (int)(r - (long long)kz * L1);
        const int gy = ky <= n1 ? ky : L1 - ky;
        const int gx = kx <= n0 ? kx : L0 - kx;
        const TI gv = ghat[((size_t)kz * (n1 + 1) + gy) * (n0 + 1) + gx];
        const CI v = f[e];
        g[e] = CO{(TO)(v.x * gv), (TO)(v.y * gv)};
    }
    __syncthreads();
    const CO* o = block_fft<TO, true>(g, h, kRowsC, px, tw_o);
    for (int e = threadIdx.x; e < kRowsC * n0; e += blockDim.x) {
        const int ri = e / n0, x = e - ri * n0;
        const long long r = r0 + ri;
        if (r < rows) out[(size_t)r * L0 + x] = o[ri * L0 + x];
    }
}

// ---------------------------------------------------------------- pass E
template <typename T, bool SELF>
__global__ void __launch_bounds__(kThreads) k_fft_z_c2r(const Cx<T>* __restrict__ spec, double* __restrict__ phi, int n0, int n1,
                                                        int n2, int L0, int L1, FftPlan pz, const Cx<T>* __restrict__ twz,
                                                        const StepState* __restrict__ st, double normFact, double coupling) {
    using C = Cx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L2 = pz.L;
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + L2;
    C* tmp = buf + 16 * L2 + 32;
    load_twiddles<T>(tw, twz, L2);
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * 32;
    // stage the half spectra of the 32 columns in tmp: [xi][k], k <= n2
    for (int e = threadIdx.x; e < 32 * (n2 + 1); e += blockDim.x) {
        const int xi = e & 31, k = e >> 5;
        const int x = x0 + xi;
        C v = C{(T)0, (T)0};
        if (x < n0) v = spec[((size_t)k * L1 + y) * L0 + x];
        if (k == 0 || k == n2) v.y = (T)0;  // the half-complex format holds no imaginary part there
        tmp[xi * (n2 + 1) + k] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 16 * L2; e += blockDim.x) {
        const int q = e / L2, k = e - q * L2;
        const C* A = tmp + (2 * q) * (n2 + 1);
        const C* B = tmp + (2 * q + 1) * (n2 + 1);
        C z;
        if (k <= n2) {
            const C a = A[k], b = B[k];
            z = C{a.x - b.y, a.y + b.x};
        } else {
            const C a = A[L2 - k], b = B[L2 - k];
            z = C{a.x + b.y, b.x - a.y};
        }
        buf[q * L2 + k] = z;
    }
    __syncthreads();
    const C* out = block_fft<T, true>(buf, tmp, 16, pz, tw);
    const double hvol = SELF ? st->hvol : 1.0;
    for (int e = threadIdx.x; e < 32 * n2; e += blockDim.x) {
        const int xi = e & 31, zz = e >> 5;
        const int x = x0 + xi;
        if (x >= n0) continue;
        const C v = out[(xi >> 1) * L2 + zz];
        double r = (double)((xi & 1) ? v.y : v.x);
        r = r * normFact;
        if (SELF) {
            r = r * hvol;
            r = r * coupling;
        }
        phi[((size_t)zz * n1 + y) * n0 + x] = r;
    }
}

// ---------------------------------------------------------------- G spectrum
// Cosine transform of every line along one axis: Y[m] = sum over the even
// extension (length 2(len-1)) of g, m in [0, len-1].  Lines are addressed as
// in[b * sb + o * so + e * se]; 32 lines per block (two per complex FFT).
template <typename TO>
__global__ void __launch_bounds__(kThreads) k_dct_lines(const double* __restrict__ in, TO* __restrict__ out, int len, int nb,
                                                        long long sb, long long so, long long se, FftPlan pl,
                                                        const double2* __restrict__ twd) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = pl.L;  // 2 (len - 1)
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* buf = tw + L;
    double2* tmp = buf + 16 * L;
    load_twiddles<double>(tw, twd, L);
    const int b0 = blockIdx.x * 32;
    const long long obase = (long long)blockIdx.y * so;
    for (int e = threadIdx.x; e < 32 * len; e += blockDim.x) {
        const int li = e & 31, m = e >> 5;
        const int b = b0 + li;
        double g = 0.0;
        if (b < nb) g = in[(long long)b * sb + obase + (long long)m * se];
        double* slot = reinterpret_cast<double*>(&buf[(li >> 1) * L + m]);
        slot[li & 1] = g;
        if (m >= 1 && m <= len - 2) {
            double* mir = reinterpret_cast<double*>(&buf[(li >> 1) * L + (L - m)]);
            mir[li & 1] = g;
        }
    }
    __syncthreads();
    const double2* o = block_fft<double, false>(buf, tmp, 16, pl, tw);
    for (int e = threadIdx.x; e < 32 * len; e += blockDim.x) {
        const int li = e & 31, m = e >> 5;
        const int b = b0 + li;
        if (b >= nb) continue;
        const double2 v = o[(li >> 1) * L + m];
        out[(long long)b * sb + obase + (long long)m * se] = (TO)((li & 1) ? v.y : v.x);
    }
}

template <typename T>
size_t smem_tile(int L, int cols) {
    return sizeof(Cx<T>) * (size_t)(L + 2 * (cols * L + 32));
}

}  // namespace

FftPlan make_plan(int L) {
    FftPlan p{};
    p.L = L;
    int m = L;
    int ns = 0;
    while (m % 16 == 0) {
        p.r[ns++] = 16;
        m /= 16;
    }
    if (m % 8 == 0) {
        p.r[ns++] = 8;
        m /= 8;
    }
    while (m % 4 == 0) {
        p.r[ns++] = 4;
        m /= 4;
    }
    while (m % 2 == 0) {
        p.r[ns++] = 2;
        m /= 2;
    }
    while (m % 3 == 0) {
        p.r[ns++] = 3;
        m /= 3;
    }
    while (m % 5 == 0) {
        p.r[ns++] = 5;
        m /= 5;
    }
    p.nst = (m == 1) ? ns : -1;
    return p;
}

size_t fft_smem_bytes(const DevBunch& b) {
    const int L[3] = {2 * b.bc.n[0], 2 * b.bc.n[1], 2 * b.bc.n[2]};
    const size_t cs = b.precision == 0 ? sizeof(double2) : sizeof(float2);
    size_t m = 0;
    for (int d = 0; d < 3; ++d) {
        m = std::max(m, cs * (size_t)(L[d] + 2 * (16 * L[d] + 32)));
        m = std::max(m, sizeof(double2) * (size_t)(L[d] + 2 * (16 * L[d] + 32)));
    }
    m = std::max(m, (sizeof(double2) + cs) * (size_t)L[0] + 2 * sizeof(double2) * (size_t)(kRowsC * L[0]));
    return m;
}

// twiddles exp(-2 pi i e / L) from long double arithmetic, rounded once
void upload_twiddles(DevBunch& b, cudaStream_t s) {
    for (int d = 0; d < 3; ++d) {
        const int L = 2 * b.bc.n[d];
        std::vector<double2> td(L);
        std::vector<float2> tf(L);
        for (int e = 0; e < L; ++e) {
            const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)e / (long double)L;
            td[e] = double2{(double)cosl(a), (double)sinl(a)};
            tf[e] = float2{(float)cosl(a), (float)sinl(a)};
        }
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
    const int L = 2 * b.bc.n[d];
    const double2* dptr = reinterpret_cast<const double2*>(b.tw[d]);
    return b.precision == 0 ? (const void*)dptr : (const void*)(dptr + L);
}

// Spectrum of the mirrored G from b.gline ((n0+1)(n1+1)(n2+1), FP64), into b.ghat.
void launch_green_transform(const DevBunch& b, cudaStream_t s) {
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long g0 = n0 + 1, g1 = n1 + 1, g2 = n2 + 1;
    const FftPlan p0 = make_plan(2 * n0), p1 = make_plan(2 * n1), p2 = make_plan(2 * n2);
    const size_t sm0 = smem_tile<double>(2 * n0, 16), sm1 = smem_tile<double>(2 * n1, 16), sm2 = smem_tile<double>(2 * n2, 16);
    const double2* tw0 = reinterpret_cast<const double2*>(b.tw[0]);
    const double2* tw1 = reinterpret_cast<const double2*>(b.tw[1]);
    const double2* tw2 = reinterpret_cast<const double2*>(b.tw[2]);
    // z lines: batch x (stride 1), outer y
    dim3 gz((unsigned)((g0 + 31) / 32), (unsigned)g1);
    k_dct_lines<double><<<gz, kThreads, sm2, s>>>(b.gline, b.gtmp, (int)g2, (int)g0, 1, g0, g0 * g1, p2, tw2);
    // y lines: batch x, outer z
    dim3 gy((unsigned)((g0 + 31) / 32), (unsigned)g2);
    k_dct_lines<double><<<gy, kThreads, sm1, s>>>(b.gtmp, b.gline, (int)g1, (int)g0, 1, g0 * g1, g0, p1, tw1);
    // x lines: batch y (stride g0), outer z
    dim3 gx((unsigned)((g1 + 31) / 32), (unsigned)g2);
    if (b.precision == 0)
        k_dct_lines<double><<<gx, kThreads, sm0, s>>>(b.gline, (double*)b.ghat, (int)g0, (int)g1, g0, g0 * g1, 1, p0, tw0);
    else
        k_dct_lines<float><<<gx, kThreads, sm0, s>>>(b.gline, (float*)b.ghat, (int)g0, (int)g1, g0, g0 * g1, 1, p0, tw0);
}

static size_t smem_conv(int L0, size_t in_bytes) {
    return (sizeof(double2) + in_bytes) * (size_t)L0 + 2 * sizeof(double2) * (size_t)(kRowsC * L0);
}

// T is the type of the forward half (A, B and the forward x transform of C);
// the inverse half (C's inverse, D, E) is FP64 in both forms.
template <typename T>
static void convolution_t(const DevBunch& b, int mode, cudaStream_t s) {
    using C = Cx<T>;
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const int L0 = 2 * n0, L1 = 2 * n1, L2 = 2 * n2;
    const FftPlan px = make_plan(L0), py = make_plan(L1), pz = make_plan(L2);
    const C* twx = reinterpret_cast<const C*>(tw_for(b, 0));
    const C* twy = reinterpret_cast<const C*>(tw_for(b, 1));
    const C* twz = reinterpret_cast<const C*>(tw_for(b, 2));
    const double2* twx_d = reinterpret_cast<const double2*>(b.tw[0]);
    const double2* twy_d = reinterpret_cast<const double2*>(b.tw[1]);
    const double2* twz_d = reinterpret_cast<const double2*>(b.tw[2]);
    C* fwd = reinterpret_cast<C*>(b.precision == 0 ? b.spec : b.spec_lo);
    double2* inv = reinterpret_cast<double2*>(b.spec);
    double normFact = 1.0;
    normFact /= L0;
    normFact /= L1;
    normFact /= L2;
    // A
    dim3 ga((unsigned)((n0 + 31) / 32), (unsigned)n1);
    k_fft_z_r2c<T><<<ga, kThreads, smem_tile<T>(L2, 16), s>>>((const T*)b.rho, fwd, n0, n1, n2, L0, L1, pz, twz);
    // B
    dim3 gb((unsigned)((n0 + 15) / 16), (unsigned)(n2 + 1));
    k_fft_y<T, false><<<gb, kThreads, smem_tile<T>(L1, 16), s>>>(fwd, n0, L0, n1, L1, py, twy);
    // C
    const long long rows = (long long)(n2 + 1) * L1;
    k_fft_x_conv<T, double><<<(unsigned)((rows + kRowsC - 1) / kRowsC), kThreads, smem_conv(L0, sizeof(C)), s>>>(
        fwd, inv, (const T*)b.ghat, n0, n1, L1, rows, px, twx, twx_d);
    // D
    k_fft_y<double, true><<<gb, kThreads, smem_tile<double>(L1, 16), s>>>(inv, n0, L0, L1, n1, py, twy_d);
    // E
    if (mode == kConvSelfField)
        k_fft_z_c2r<double, true><<<ga, kThreads, smem_tile<double>(L2, 16), s>>>(inv, b.phi, n0, n1, n2, L0, L1, pz, twz_d,
                                                                                   b.st, normFact, b.bc.coupling);
    else
        k_fft_z_c2r<double, false><<<ga, kThreads, smem_tile<double>(L2, 16), s>>>(inv, b.phi, n0, n1, n2, L0, L1, pz, twz_d,
                                                                                    b.st, normFact, b.bc.coupling);
}

void launch_convolution(const DevBunch& b, int mode, cudaStream_t s) {
    if (b.precision == 0)
        convolution_t<double>(b, mode, s);
    else
        convolution_t<float>(b, mode, s);
}

void fft_set_smem_limits() {
    const int big = 227 * 1024;
    cudaFuncSetAttribute(k_fft_z_r2c<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_fft_z_r2c<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_fft_y<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_fft_y<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_fft_y<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_fft_x_conv<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_fft_x_conv<float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_fft_z_c2r<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_fft_z_c2r<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_dct_lines<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_dct_lines<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
}

}  // namespace sc
