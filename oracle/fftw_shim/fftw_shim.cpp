/*
 * Test infrastructure (oracle side only; never linked into the product).
 *
 * Project-written implementation of the FFTW3-float entry points MEGADOCK's CPU
 * path calls (src/fft_process.cpp:188-202 plan/alloc, :386-388 execute,
 * :822-823 destroy; src/fft_process.h:159-161 free/cleanup).  libfftw3f is not
 * available on this image, so this file stands in for it when the reference's
 * own CPU sources are compiled as the oracle.
 *
 * Transform: unnormalised 3D complex DFT, row-major [n0][n1][n2], out-of-place,
 *   out[k] = sum_j in[j] * exp(sign * 2*pi*i * <j,k/n>)  (sign = -1 forward).
 * Method: separable per-axis 1D transforms; each 1D transform is an iterative
 * Stockham autosort FFT (Govindaraju et al., SC'08 formulation) over the prime
 * factorisation of n (radix 4 first, then 2, 3, 5, 7, ... with a direct DFT for
 * each radix), twiddles computed in double precision.
 *
 * MD_SHIM_FFT=fp32 (default): float arithmetic (stand-in for FFTW's float path).
 * MD_SHIM_FFT=fp64: double arithmetic, rounded to float once on output.
 * Thread safety: plans are immutable after creation; every execute call uses
 * its own scratch, so concurrent execution of distinct plans is safe (the
 * reference executes one plan per OpenMP thread concurrently).
 */
#include "fftw3.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

template <typename T>
struct Cx {
    T re, im;
};

struct Stage {
    int radix;
    int ns;                       // product of the radices of earlier stages
    std::vector<double> tw_re;    // [(j % ns) * radix + r]
    std::vector<double> tw_im;
    std::vector<double> w_re;     // W_radix^m, m in [0, radix)
    std::vector<double> w_im;
};

struct Axis {
    int n;
    std::vector<Stage> stages;
};

static void build_axis(Axis &ax, int n, int sign) {
    ax.n = n;
    std::vector<int> rad;
    int m = n;
    while (m % 4 == 0) { rad.push_back(4); m /= 4; }
    while (m % 2 == 0) { rad.push_back(2); m /= 2; }
    for (int p = 3; m > 1; p += 2) {
        while (m % p == 0) { rad.push_back(p); m /= p; }
    }
    int ns = 1;
    for (int r : rad) {
        Stage st;
        st.radix = r;
        st.ns = ns;
        st.tw_re.resize((size_t)ns * r);
        st.tw_im.resize((size_t)ns * r);
        for (int jm = 0; jm < ns; ++jm) {
            for (int q = 0; q < r; ++q) {
                const double ang = sign * 2.0 * M_PI * (double)jm * q / ((double)ns * r);
                st.tw_re[(size_t)jm * r + q] = std::cos(ang);
                st.tw_im[(size_t)jm * r + q] = std::sin(ang);
            }
        }
        st.w_re.resize(r);
        st.w_im.resize(r);
        for (int q = 0; q < r; ++q) {
            const double ang = sign * 2.0 * M_PI * (double)q / r;
            st.w_re[q] = std::cos(ang);
            st.w_im[q] = std::sin(ang);
        }
        ax.stages.push_back(st);
        ns *= r;
    }
}

// One 1D transform of a contiguous line.  Result ends in `a` (copied if needed).
template <typename T>
static void fft_line(const Axis &ax, int sign, Cx<T> *a, Cx<T> *b) {
    const int n = ax.n;
    Cx<T> *src = a, *dst = b;
    Cx<T> v[64], o[64];
    for (const Stage &st : ax.stages) {
        const int R = st.radix;
        const int ns = st.ns;
        const int nr = n / R;
        std::vector<Cx<T>> big;
        Cx<T> *vv = v, *oo = o;
        if (R > 64) {
            big.resize(2 * (size_t)R);
            vv = big.data();
            oo = big.data() + R;
        }
        for (int j = 0; j < nr; ++j) {
            const int jm = j % ns;
            for (int q = 0; q < R; ++q) {
                const Cx<T> x = src[j + q * nr];
                const T wr = (T)st.tw_re[(size_t)jm * R + q];
                const T wi = (T)st.tw_im[(size_t)jm * R + q];
                vv[q].re = x.re * wr - x.im * wi;
                vv[q].im = x.re * wi + x.im * wr;
            }
            if (R == 4) {
                const T t0r = vv[0].re + vv[2].re, t0i = vv[0].im + vv[2].im;
                const T t1r = vv[0].re - vv[2].re, t1i = vv[0].im - vv[2].im;
                const T t2r = vv[1].re + vv[3].re, t2i = vv[1].im + vv[3].im;
                const T dr = vv[1].re - vv[3].re, di = vv[1].im - vv[3].im;
                // (v1 - v3) * (sign * i)
                const T t3r = -(T)sign * di, t3i = (T)sign * dr;
                oo[0].re = t0r + t2r; oo[0].im = t0i + t2i;
                oo[2].re = t0r - t2r; oo[2].im = t0i - t2i;
                oo[1].re = t1r + t3r; oo[1].im = t1i + t3i;
                oo[3].re = t1r - t3r; oo[3].im = t1i - t3i;
            } else if (R == 2) {
                oo[0].re = vv[0].re + vv[1].re; oo[0].im = vv[0].im + vv[1].im;
                oo[1].re = vv[0].re - vv[1].re; oo[1].im = vv[0].im - vv[1].im;
            } else {
                for (int k = 0; k < R; ++k) {
                    T sr = 0, si = 0;
                    for (int q = 0; q < R; ++q) {
                        const int m = (int)(((long long)q * k) % R);
                        const T wr = (T)st.w_re[m], wi = (T)st.w_im[m];
                        sr += vv[q].re * wr - vv[q].im * wi;
                        si += vv[q].re * wi + vv[q].im * wr;
                    }
                    oo[k].re = sr;
                    oo[k].im = si;
                }
            }
            const int idxd = (j / ns) * ns * R + jm;
            for (int q = 0; q < R; ++q) dst[idxd + q * ns] = oo[q];
        }
        Cx<T> *t = src; src = dst; dst = t;
    }
    if (src != a) std::memcpy(a, src, sizeof(Cx<T>) * n);
}

// Transform every line of one axis of a row-major 3D array in place.
template <typename T>
static void fft_axis(const Axis &ax, int sign, Cx<T> *data, const int dims[3], int axis) {
    const int n = dims[axis];
    size_t stride = 1;
    for (int d = axis + 1; d < 3; ++d) stride *= dims[d];
    size_t outer = 1;
    for (int d = 0; d < axis; ++d) outer *= dims[d];
    const int block = (stride >= 16) ? 16 : (int)stride;
    std::vector<Cx<T>> buf((size_t)n * block), tmp(n);
    for (size_t o = 0; o < outer; ++o) {
        Cx<T> *base = data + o * (size_t)n * stride;
        for (size_t s0 = 0; s0 < stride; s0 += block) {
            const int nb = (int)((stride - s0) < (size_t)block ? (stride - s0) : (size_t)block);
            for (int e = 0; e < n; ++e)
                for (int l = 0; l < nb; ++l) buf[(size_t)l * n + e] = base[(size_t)e * stride + s0 + l];
            for (int l = 0; l < nb; ++l) fft_line(ax, sign, &buf[(size_t)l * n], tmp.data());
            for (int e = 0; e < n; ++e)
                for (int l = 0; l < nb; ++l) base[(size_t)e * stride + s0 + l] = buf[(size_t)l * n + e];
        }
    }
}

static bool use_fp64() {
    const char *e = std::getenv("MD_SHIM_FFT");
    return e && std::strcmp(e, "fp64") == 0;
}

}  // namespace

struct fftwf_plan_s {
    int dims[3];
    int sign;
    fftwf_complex *in;
    fftwf_complex *out;
    Axis axes[3];
};

extern "C" {

fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags) {
    (void)flags;
    if (n0 <= 0 || n1 <= 0 || n2 <= 0) return nullptr;
    fftwf_plan p = new fftwf_plan_s;
    p->dims[0] = n0;
    p->dims[1] = n1;
    p->dims[2] = n2;
    p->sign = sign < 0 ? -1 : 1;
    p->in = in;
    p->out = out;
    for (int d = 0; d < 3; ++d) build_axis(p->axes[d], p->dims[d], p->sign);
    return p;
}

void fftwf_execute(const fftwf_plan p) {
    if (!p) return;
    const size_t total = (size_t)p->dims[0] * p->dims[1] * p->dims[2];
    if (use_fp64()) {
        std::vector<Cx<double>> w(total);
        for (size_t i = 0; i < total; ++i) {
            w[i].re = p->in[i][0];
            w[i].im = p->in[i][1];
        }
        for (int d = 2; d >= 0; --d) fft_axis<double>(p->axes[d], p->sign, w.data(), p->dims, d);
        for (size_t i = 0; i < total; ++i) {
            p->out[i][0] = (float)w[i].re;
            p->out[i][1] = (float)w[i].im;
        }
    } else {
        Cx<float> *o = reinterpret_cast<Cx<float> *>(p->out);
        if ((void *)p->out != (void *)p->in) std::memcpy(p->out, p->in, sizeof(fftwf_complex) * total);
        for (int d = 2; d >= 0; --d) fft_axis<float>(p->axes[d], p->sign, o, p->dims, d);
    }
}

void fftwf_destroy_plan(fftwf_plan p) { delete p; }

void *fftwf_malloc(size_t n) {
    void *ptr = nullptr;
    if (posix_memalign(&ptr, 64, n ? n : 1) != 0) return nullptr;
    return ptr;
}

void fftwf_free(void *p) { std::free(p); }

void fftwf_cleanup(void) {}

}  // extern "C"
