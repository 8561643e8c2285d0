// fft.cuh -- shared-memory Stockham FFT engine (FP64 complex).
//
// The reference diagonalises the Poisson operator with library FFTs
// (AbstractFFTs -> FFTW/cuFFT: rfft along x, fft along z, fft along y for
// periodic boxes; src/poisson.jl:80-83,115-116).  Here every transform runs
// inside the kernel that also does the surrounding stencil or solve work: a
// CTA stages L lines in shared memory and all of its threads run the
// mixed-radix Stockham autosort stages on them, so a line is read from and
// written to HBM once per pass.
//
// Conventions (AbstractFFTs): forward uses exp(-2 pi i jk/n) unscaled; the
// inverse uses exp(+2 pi i jk/n); scaling is applied by the caller.
//
// Data in shared memory: element e of line l sits at buf[l*ls + e*es]; the
// stages ping-pong between two such buffers.
// The twiddle table tw[t] = exp(-2 pi i t/n), t = 0..n-1, is also in shared
// memory; it is computed on the host in long double and rounded once.
#pragma once
#include <cuda_runtime.h>

namespace dnsb {

constexpr int FFT_MAX_STAGES = 24;

struct FFTPlan {
  int n;
  int nst;
  int radix[FFT_MAX_STAGES];
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// R-point DFT in registers (R = 2, 3, 4, 5, 8), forward
// y_s = sum_q v_q W_R^{qs} with W_R = e^{-2 pi i/R}; INV uses conj(W_R).
// The constants are cos/sin of 2 pi/3, 2 pi/5, 4 pi/5.
template <int R, bool INV>
__device__ __forceinline__ void dft_small(double2 (&v)[R]) {
  // multiply by -i (forward) or +i (inverse)
  auto rot = [](double2 t) { return INV ? make_double2(-t.y, t.x) : make_double2(t.y, -t.x); };
  if constexpr (R == 2) {
    double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 3) {
    constexpr double s3 = 0.86602540378443864676;  // sin(2 pi/3)
    const double2 t1 = cadd(v[1], v[2]);
    const double2 t2 = rot(cscale(csub(v[1], v[2]), s3));
    const double2 m = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, t2);
    v[2] = csub(m, t2);
  } else if constexpr (R == 4) {
    double2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    double2 c = cadd(v[1], v[3]);
    double2 d = rot(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  } else if constexpr (R == 8) {
    // two 4-point DFTs of the even and odd samples, combined with W_8^k
    constexpr double h = 0.70710678118654752440;  // sqrt(1/2)
    double2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft_small<4, INV>(e);
    dft_small<4, INV>(o);
    const double2 o1 = INV ? make_double2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                           : make_double2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    const double2 o2 = rot(o[2]);
    const double2 o3 = INV ? make_double2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                           : make_double2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  } else if constexpr (R == 5) {
    constexpr double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    constexpr double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
    const double2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    const double2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    const double2 m1 = make_double2(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    const double2 m2 = make_double2(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    const double2 n1 = rot(make_double2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    const double2 n2 = rot(make_double2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    v[0] = cadd(v[0], cadd(a1, a2));
    v[1] = cadd(m1, n1);
    v[4] = csub(m1, n1);
    v[2] = cadd(m2, n2);
    v[3] = csub(m2, n2);
  }
}

// One Stockham stage of radix R over L lines of length n (Ns = product of
// the radices already applied), from buffer `in` to buffer `out` (both in
// shared memory, same layout).  All threads of the CTA take butterflies in
// turn; one barrier ends the stage.  jfast: consecutive threads take
// consecutive butterflies of one line (use when es == 1); otherwise
// consecutive threads take consecutive lines.
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(const double2 *__restrict__ in, double2 *__restrict__ out,
                                          int n, int Ns, int L, int es, int ls, bool jfast,
                                          const double2 *__restrict__ tw) {
  const int nb = n / R;
  const int total = nb * L;
  const int stride_tw = n / (Ns * R);
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    int l, j;
    if (jfast) { l = b / nb; j = b - l * nb; }
    else { j = b / L; l = b - j * L; }
    const double2 *src = in + l * ls;
    double2 *dst = out + l * ls;
    const int k = j % Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = src[(j + r * nb) * es];
    if (k != 0) {
#pragma unroll
      for (int r = 1; r < R; r++) {
        double2 w = tw[k * r * stride_tw];
        if (INV) w = cconj(w);
        v[r] = cmul(v[r], w);
      }
    }
    dft_small<R, INV>(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) dst[(base + r * Ns) * es] = v[r];
  }
  __syncthreads();
}

// Full transform of L lines; ping-pongs between a and b and returns the
// buffer that holds the result.  The caller must have synchronised after
// filling a.
template <bool INV>
__device__ double2 *fft_lines(double2 *a, double2 *b, const FFTPlan &p, int L, int es, int ls,
                              bool jfast, const double2 *__restrict__ tw) {
  int Ns = 1;
  for (int s = 0; s < p.nst; s++) {
    const int R = p.radix[s];
    switch (R) {
      case 2: fft_stage<2, INV>(a, b, p.n, Ns, L, es, ls, jfast, tw); break;
      case 3: fft_stage<3, INV>(a, b, p.n, Ns, L, es, ls, jfast, tw); break;
      case 4: fft_stage<4, INV>(a, b, p.n, Ns, L, es, ls, jfast, tw); break;
      case 5: fft_stage<5, INV>(a, b, p.n, Ns, L, es, ls, jfast, tw); break;
      case 8: fft_stage<8, INV>(a, b, p.n, Ns, L, es, ls, jfast, tw); break;
      default: break;  // rejected on the host
    }
    Ns *= R;
    double2 *t = a;
    a = b;
    b = t;
  }
  return a;
}

// Stages that read their inputs from, or write their outputs to, global
// memory through functors, so that the first stage loads straight into
// registers (R independent loads in flight per butterfly, no staging copy)
// and the last stage stores straight from registers.
// ld(l, e) returns element e of line l; st(l, e, v) stores it.
template <int R, bool INV, class Ld, class St>
__device__ __forceinline__ void fft_stage_io(Ld ld, const double2 *__restrict__ in,
                                             double2 *__restrict__ out, St st, bool gin,
                                             bool gout, int n, int Ns, int L, int es, int ls,
                                             bool jfast, const double2 *__restrict__ tw) {
  const int nb = n / R;
  const int total = nb * L;
  const int stride_tw = n / (Ns * R);
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    int l, j;
    if (jfast) { l = b / nb; j = b - l * nb; }
    else { j = b / L; l = b - j * L; }
    const int k = j % Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = gin ? ld(l, j + r * nb) : in[l * ls + (j + r * nb) * es];
    if (k != 0) {
#pragma unroll
      for (int r = 1; r < R; r++) {
        double2 w = tw[k * r * stride_tw];
        if (INV) w = cconj(w);
        v[r] = cmul(v[r], w);
      }
    }
    dft_small<R, INV>(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) {
      if (gout) st(l, base + r * Ns, v[r]);
      else out[l * ls + (base + r * Ns) * es] = v[r];
    }
  }
  __syncthreads();
}

template <bool INV, class Ld, class St>
__device__ __forceinline__ void fft_stage_io_any(int R, Ld ld, const double2 *in, double2 *out,
                                                 St st, bool gin, bool gout, int n, int Ns, int L,
                                                 int es, int ls, bool jfast,
                                                 const double2 *__restrict__ tw) {
  switch (R) {
    case 2: fft_stage_io<2, INV>(ld, in, out, st, gin, gout, n, Ns, L, es, ls, jfast, tw); break;
    case 3: fft_stage_io<3, INV>(ld, in, out, st, gin, gout, n, Ns, L, es, ls, jfast, tw); break;
    case 4: fft_stage_io<4, INV>(ld, in, out, st, gin, gout, n, Ns, L, es, ls, jfast, tw); break;
    case 5: fft_stage_io<5, INV>(ld, in, out, st, gin, gout, n, Ns, L, es, ls, jfast, tw); break;
    case 8: fft_stage_io<8, INV>(ld, in, out, st, gin, gout, n, Ns, L, es, ls, jfast, tw); break;
    default: break;
  }
}

// Transform of L lines in which the first stage reads with ld (when
// load_global, else from a) and the last stage writes with st (when
// store_global, else to shared memory); the stages between ping-pong in
// shared memory (a, b with layout es/ls).  Returns the shared buffer that
// holds the result when !store_global.  The twiddle table must be in place
// (and synchronised) before the call.
template <bool INV, class Ld, class St>
__device__ double2 *fft_lines_io(Ld ld, St st, double2 *a, double2 *b, const FFTPlan &p, int L,
                                 int es, int ls, bool jfast, const double2 *__restrict__ tw,
                                 bool load_global, bool store_global) {
  int Ns = 1;
  for (int s = 0; s < p.nst; s++) {
    const int R = p.radix[s];
    const bool gin = load_global && s == 0, gout = store_global && s == p.nst - 1;
    fft_stage_io_any<INV>(R, ld, a, b, st, gin, gout, p.n, Ns, L, es, ls, jfast, tw);
    Ns *= R;
    double2 *t = a;
    a = b;
    b = t;
  }
  return a;
}

// Host-side plan: radices 8 first, then 4, 2, 3, 5.  Returns false
// when n has another prime factor.
inline bool make_fft_plan(int n, FFTPlan &p) {
  p.n = n;
  p.nst = 0;
  int m = n;
  while (m % 8 == 0 && p.nst < FFT_MAX_STAGES) { p.radix[p.nst++] = 8; m /= 8; }
  while (m % 4 == 0 && p.nst < FFT_MAX_STAGES) { p.radix[p.nst++] = 4; m /= 4; }
  const int primes[] = {2, 3, 5};
  for (int q : primes)
    while (m % q == 0 && p.nst < FFT_MAX_STAGES) { p.radix[p.nst++] = q; m /= q; }
  return m == 1 && n >= 1;
}

}  // namespace dnsb
