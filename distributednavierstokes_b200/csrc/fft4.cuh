// fft4.cuh -- four-step FFT with register-resident sub-transforms.
//
// A line of length N = N1*N2 is transformed as
//   step 1: thread (line, j2) loads x[j1*N2 + j2], j1 = 0..N1-1, does an
//           N1-point FFT in registers, multiplies by W_N^(j2*k1) and writes
//           the N1 results to a shared-memory transpose buffer;
//   step 2: thread (line, k1) reads its N2 values, does an N2-point FFT in
//           registers and emits X[k1 + N1*k2], k2 = 0..N2-1.
// Each element crosses shared memory once (one write, one read) instead of
// once per radix stage, which keeps the transform kernels HBM-bound.  Loads
// of step 1 (strided by N2 within a line) and stores of step 2 (strided by
// N1) are coalesced across threads.  The register FFTs are mixed-radix
// Stockham (radices 8, 4, 2, 3, 5) with all indices known at compile time.
// Twiddles come from the kernel's table tw[t] = exp(-2 pi i t/N).
#pragma once
#include "fft.cuh"

namespace dnsb {

__host__ __device__ constexpr int reg_radix(int m) {
  return m % 8 == 0 ? 8 : m % 4 == 0 ? 4 : m % 2 == 0 ? 2 : m % 3 == 0 ? 3 : m % 5 == 0 ? 5 : m;
}

// Stages NS.. of an N-point FFT of v (in place); twiddle W_N^a = tw[a * ts]
template <int N, int NS, bool INV>
__device__ __forceinline__ void reg_fft_stages(double2 (&v)[N], const double2 *__restrict__ tw,
                                               int ts) {
  if constexpr (NS < N) {
    constexpr int R = reg_radix(N / NS);
    static_assert(R == 2 || R == 3 || R == 4 || R == 5 || R == 8, "unsupported radix");
    constexpr int NB = N / R;
    double2 t[N];
#pragma unroll
    for (int j = 0; j < NB; j++) {
      const int k = j % NS;
      double2 a[R];
#pragma unroll
      for (int r = 0; r < R; r++) a[r] = v[j + r * NB];
      if (k != 0) {
#pragma unroll
        for (int r = 1; r < R; r++) {
          double2 w = tw[(k * r * (N / (NS * R))) * ts];
          if (INV) w = cconj(w);
          a[r] = cmul(a[r], w);
        }
      }
      dft_small<R, INV>(a);
      const int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) t[base + r * NS] = a[r];
    }
#pragma unroll
    for (int i = 0; i < N; i++) v[i] = t[i];
    reg_fft_stages<N, NS * R, INV>(v, tw, ts);
  }
}

template <int N, bool INV>
__device__ __forceinline__ void reg_fft(double2 (&v)[N], const double2 *__restrict__ tw, int ts) {
  reg_fft_stages<N, 1, INV>(v, tw, ts);
}

// Row pitch (complex) of the transpose buffer: N2 padded to an odd count.
template <int N2>
__host__ __device__ constexpr int fft4_pitch() {
  return (N2 % 2 == 0) ? N2 + 1 : N2;
}

// Shared-memory complex values used by fft4_lines for L lines.
template <int N1, int N2>
__host__ __device__ constexpr int fft4_buf(int L) {
  return L * N1 * fft4_pitch<N2>();
}

// Four-step transform of L lines of length N1*N2.  ld(l, e) returns input
// element e of line l; st(l, e, v) stores output element e.  buf holds
// fft4_buf<N1,N2>(L) values; tw holds N1*N2 twiddles (exp(-2 pi i t/N)).
// All loads of step 1 precede (barrier) all stores of step 2, so st may
// overwrite what ld reads.  Ends with a barrier.
template <int N1, int N2, bool INV, class Ld, class St>
__device__ __forceinline__ void fft4_lines(Ld ld, St st, double2 *buf, int L,
                                           const double2 *__restrict__ tw) {
  constexpr int P = fft4_pitch<N2>();
  const int nth = blockDim.x;
  // step 1: N1-point transforms of the stride-N2 subsequences
  for (int it = threadIdx.x; it < L * N2; it += nth) {
    const int l = it / N2, j2 = it - l * N2;
    double2 v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) v[j1] = ld(l, j1 * N2 + j2);
    reg_fft<N1, INV>(v, tw, N2);
    double2 *row = buf + l * N1 * P + j2;
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) {
      double2 w = tw[j2 * k1];
      if (INV) w = cconj(w);
      row[k1 * P] = k1 == 0 ? v[0] : cmul(v[k1], w);
    }
  }
  __syncthreads();
  // step 2: N2-point transforms across the subsequences
  for (int it = threadIdx.x; it < L * N1; it += nth) {
    const int l = it / N1, k1 = it - l * N1;
    double2 v[N2];
    const double2 *col = buf + l * N1 * P + k1 * P;
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++) v[j2] = col[j2];
    reg_fft<N2, INV>(v, tw, N1);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) st(l, k1 + N1 * k2, v[k2]);
  }
  __syncthreads();
}

// Host-side choice of the (N1, N2) split for the lengths with a specialised
// kernel; returns false when the generic Stockham kernels must be used.
inline bool fft4_split(int n, int &n1, int &n2) {
  switch (n) {
    case 384: n1 = 16; n2 = 24; return true;
    case 256: n1 = 16; n2 = 16; return true;
    case 192: n1 = 16; n2 = 12; return true;
    case 128: n1 = 16; n2 = 8; return true;
    case 96: n1 = 8; n2 = 12; return true;
    case 64: n1 = 8; n2 = 8; return true;
    case 48: n1 = 8; n2 = 6; return true;
    case 32: n1 = 8; n2 = 4; return true;
    default: return false;
  }
}

}  // namespace dnsb
