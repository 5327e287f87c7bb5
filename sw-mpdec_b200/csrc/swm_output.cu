// swm_output.cu -- WriteSolutionToDisk / WriteMeshToDisk on the device (sm_100a).
//
// The reference writes every value with the edit descriptor (SP,ES21.14E2): sign,
// one digit, a point, 14 digits, E, exponent sign, two exponent digits
// (output.f90:263-301,355-358).  Formatting is the expensive part of its output at
// 2048^2 (25 M values per file), so here each value is formatted by one thread into
// a fixed-width line buffer that is copied to the host once.
//
// Digits are exact: a finite x = M 2^E is the integer C = M 5^k (E = -k < 0) or
// C = M 2^E (E >= 0) times 10^-k; C's decimal expansion (repeated division by 10^9)
// is rounded to 15 significant digits, ties to even (C's printf rounding of the
// exact binary value).  Exponents beyond two digits print 21 asterisks, as a
// Fortran Ew.dEe field that cannot hold its exponent does; NaN and infinities are
// right-justified words.
#include <cstdint>

#include "swm_kernels.cuh"

namespace swm {

namespace {

constexpr int kLimbs = 84;  // 32-bit limbs: M 5^1074 < 2^2547 and M 2^971 < 2^1024

// c[0..n) *= m (m < 2^32); returns the new limb count
__device__ __forceinline__ int big_mul(uint32_t* c, int n, uint32_t m) {
  uint64_t carry = 0;
  for (int i = 0; i < n; ++i) {
    const uint64_t t = (uint64_t)c[i] * m + carry;
    c[i] = (uint32_t)t;
    carry = t >> 32;
  }
  if (carry) c[n++] = (uint32_t)carry;
  return n;
}

// c[0..n) /= d in place; returns the remainder, *n drops leading zero limbs
__device__ __forceinline__ uint32_t big_div(uint32_t* c, int* n, uint32_t d) {
  uint64_t rem = 0;
  for (int i = *n - 1; i >= 0; --i) {
    const uint64_t cur = (rem << 32) | c[i];
    c[i] = (uint32_t)(cur / d);
    rem = cur % d;
  }
  while (*n > 0 && c[*n - 1] == 0) --*n;
  return (uint32_t)rem;
}

__device__ void put_word(char* out, const char* w, int len) {  // right-justified in 21
  for (int i = 0; i < 21; ++i) out[i] = ' ';
  for (int i = 0; i < len; ++i) out[21 - len + i] = w[i];
}

}  // namespace

// x as (SP,ES21.14E2) into out[0..21)
__device__ void format_es21(double x, char* out) {
  const uint64_t bits = (uint64_t)__double_as_longlong(x);
  const bool neg = bits >> 63;
  const int be = (int)((bits >> 52) & 0x7ff);
  uint64_t M = bits & ((1ull << 52) - 1);
  if (be == 0x7ff) {
    if (M) {
      put_word(out, "NaN", 3);
    } else {
      put_word(out, neg ? "-Infinity" : "+Infinity", 9);
    }
    return;
  }
  char digs[16];
  int e10 = 0;
  if (be == 0 && M == 0) {
    for (int i = 0; i < 15; ++i) digs[i] = '0';
  } else {
    int E;
    if (be == 0) {
      E = -1074;
    } else {
      M |= 1ull << 52;
      E = be - 1075;
    }
    while (E < 0 && !(M & 1)) {  // fewer factors of 5 to carry
      M >>= 1;
      ++E;
    }
    uint32_t c[kLimbs];
    c[0] = (uint32_t)M;
    c[1] = (uint32_t)(M >> 32);
    int n = c[1] ? 2 : 1;
    int k = 0;
    if (E >= 0) {  // C = M 2^E: whole limbs, then bits
      const int w = E / 32, b = E % 32;
      for (int i = n - 1; i >= 0; --i) c[i + w] = c[i];
      for (int i = 0; i < w; ++i) c[i] = 0;
      n += w;
      if (b) n = big_mul(c, n, 1u << b);
    } else {  // C = M 5^k
      k = -E;
      int r = k;
      for (; r >= 13; r -= 13) n = big_mul(c, n, 1220703125u);  // 5^13
      uint32_t p = 1;
      for (; r > 0; --r) p *= 5;
      if (p > 1) n = big_mul(c, n, p);
    }
    // decimal chunks of C, least significant first
    uint32_t ch[kLimbs * 32 / 29 + 2];
    int nch = 0;
    while (n > 0) ch[nch++] = big_div(c, &n, 1000000000u);
    int top = 0;  // digits in the most significant chunk
    for (uint32_t t = ch[nch - 1]; t; t /= 10) ++top;
    const int nd = 9 * (nch - 1) + top;
    e10 = nd - 1 - k;
    // the first 16 digits and whether anything non-zero follows
    char d16[16];
    int got = 0;
    bool sticky = false;
    for (int q = nch - 1; q >= 0; --q) {
      const int len = (q == nch - 1) ? top : 9;
      uint32_t v = ch[q];
      char tmp[9];
      for (int i = len - 1; i >= 0; --i) {
        tmp[i] = (char)('0' + v % 10);
        v /= 10;
      }
      for (int i = 0; i < len; ++i) {
        if (got < 16)
          d16[got++] = tmp[i];
        else if (tmp[i] != '0')
          sticky = true;
      }
    }
    for (; got < 16; ++got) d16[got] = '0';
    uint64_t D = 0;
    for (int i = 0; i < 15; ++i) D = D * 10 + (uint64_t)(d16[i] - '0');
    const int r = d16[15] - '0';
    if (r > 5 || (r == 5 && (sticky || (D & 1)))) {
      ++D;
      if (D == 1000000000000000ull) {
        D = 100000000000000ull;
        ++e10;
      }
    }
    for (int i = 14; i >= 0; --i) {
      digs[i] = (char)('0' + D % 10);
      D /= 10;
    }
  }
  if (e10 > 99 || e10 < -99) {
    for (int i = 0; i < 21; ++i) out[i] = '*';
    return;
  }
  out[0] = neg ? '-' : '+';
  out[1] = digs[0];
  out[2] = '.';
  for (int i = 1; i < 15; ++i) out[2 + i] = digs[i];
  out[17] = 'E';
  out[18] = e10 < 0 ? '-' : '+';
  const int ae = e10 < 0 ? -e10 : e10;
  out[19] = (char)('0' + ae / 10);
  out[20] = (char)('0' + ae % 10);
}

namespace {

// One line per cell (jj outer, ii inner): ncoord (0 or 2) barycentre coordinates
// then nval values, each as ES21.14E2 followed by `sep` spaces, then '\n'.  Data values with |v| < 1e-70 print as 0
// (output.f90:289-295).
__global__ void __launch_bounds__(256) lines_kernel(const OutLines a) {
  const int per = a.ncoord + a.nval;
  const long long total = (long long)a.nx * a.ny * per;
  const int lw = per * (21 + a.sep) + 1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long cell = t / per;
    const int slot = (int)(t % per);
    const int i = (int)(cell % a.nx), j = (int)(cell / a.nx);
    double v;
    if (slot < a.ncoord) {
      // MeshBary = MeshNodes(ii-1,jj-1) + 0.5 Mesh_DX (mesh.f90:64-70)
      v = slot == 0 ? (a.x0 + ((double)i) * a.dx) + 0.5 * a.dx
                    : (a.y0 + ((double)j) * a.dy) + 0.5 * a.dy;
    } else {
      const double* p = a.val[slot - a.ncoord];
      v = p ? p[cell] : 0.0;
      if (a.zero_small && fabs(v) < 1.e-70) v = 0.0;
    }
    char* o = a.out + cell * lw + slot * (21 + a.sep);
    format_es21(v, o);
    for (int s = 0; s < a.sep; ++s) o[21 + s] = ' ';
    if (slot == per - 1) o[21 + a.sep] = '\n';
  }
}

// V = ConsToPrim(U) of planes (equation.f90:912-945), the reference's rounding
__global__ void prim_kernel(const double* h, const double* hu, const double* hv, double* u,
                            double* v, int n) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double uu, vv;
    cons_to_prim<true>(h[c], hu[c], hv[c], uu, vv);
    u[c] = uu;
    v[c] = vv;
  }
}

__global__ void format_kernel(const double* x, int n, char* out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    format_es21(x[k], out + 21 * (size_t)k);
}

int grid_for(long long work) {
  long long b = (work + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}

}  // namespace

size_t out_line_width(const OutLines& a) { return (size_t)(a.ncoord + a.nval) * (21 + a.sep) + 1; }

cudaError_t launch_out_lines(const OutLines& a, cudaStream_t s) {
  lines_kernel<<<grid_for((long long)a.nx * a.ny * (a.ncoord + a.nval)), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_prim(const double* h, const double* hu, const double* hv, double* u, double* v,
                        int n, cudaStream_t s) {
  prim_kernel<<<grid_for(n), 256, 0, s>>>(h, hu, hv, u, v, n);
  return cudaGetLastError();
}

cudaError_t launch_format_values(const double* x, int n, char* out, cudaStream_t s) {
  format_kernel<<<grid_for(n), 256, 0, s>>>(x, n, out);
  return cudaGetLastError();
}

}  // namespace swm
