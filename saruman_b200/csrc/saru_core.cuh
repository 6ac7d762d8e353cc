// saru_core.cuh -- per-candidate banded alignment core (device code).
//
// One candidate = read r[0..m) against genome window g[0..L), DP matrix
// D[0..L][0..m] (row = window position, column = read position) with the
// reference's rules (src/cuda-functions.cu:413-497):
//   D[0][j] = j;  D[i][0] = max(0, i - 2*so);
//   D[i][j] = min(D[i-1][j-1] + (g[i-1] != r[j-1]),  D[i][j-1] + 1,
//                 D[i-1][j] + 1 - [j == m && i-1 >= L - 2*eo])
// for the unit costs match = 0, mismatch = 1.
//
// Fill: bit-parallel over a diagonal band.  For read column j the band holds
// rows j - k + b for bit b in [0, BITS) (BITS = 32 or 64).  Every cell whose
// value is <= k lies on a diagonal d = i - j in [-k, 2*so + k] (the value of
// a cell is at least j - i, and at least i - j - 2*so off the last column),
// so this band holds all of them whenever 2*so + k <= BITS - 1 - k.  Each
// column is one step of the Myers/Hyyro vertical-delta recurrence, the
// previous column's vectors shifted down one bit to follow the diagonal.
// Cells outside the band enter as "+1 from a neighbour" (the cost of a real
// path), so every band value is an upper bound and is exact when <= k.
// Rows above row 0 are virtual (D[-r][j] = j + r), which gives row 0 = j.
//
// The last read column has free vertical moves below row L - 2*eo and is
// evaluated with explicit values from the band of column m-1.
//
// For every band cell the traceback decision of the reference
// (src/cuda-functions.cu:215-276) is recorded as 2 bits:
//   DIAG if D[i-1][j-1] + 1 == v, or D[i-1][j-1] == v and the bytes match
//   UP   else if D[i-1][j] + 1 - corr == v
//   LEFT else if D[i][j-1] + 1 == v
//   STOP otherwise
// with corr = 1 on the last column below row L - 2eo and, when so != 0, on
// the first column for rows <= 2so + 3 (src/cuda-functions.cu:181-190).
// The traceback only visits cells with value <= k, where these decisions
// equal the reference's: a neighbour that is > k (exact or bound) fails the
// equality tests either way.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define SARU_HD __host__ __device__ __forceinline__
#else
#define SARU_HD inline
#endif

namespace saru {

enum : int { OP_STOP = 0, OP_DIAG = 1, OP_UP = 2, OP_LEFT = 3 };

// read-byte classes: A C G T, then up to MAX_EXTRA other bytes of the read
constexpr int MAX_EXTRA = 2;
constexpr int NCODES = 4 + MAX_EXTRA;

SARU_HD uint32_t fshr32(uint32_t lo, uint32_t hi, uint32_t s) {
#if defined(__CUDA_ARCH__)
  return __funnelshift_r(lo, hi, s);
#else
  s &= 31;
  return s ? (lo >> s) | (hi << (32 - s)) : lo;
#endif
}

template <typename T>
SARU_HD T lowmask(int n) {
  constexpr int BITS = int(sizeof(T) * 8);
  return n <= 0 ? T(0) : (n >= BITS ? ~T(0) : ((T(1) << n) - T(1)));
}

// Word arrays are addressed through P, either a plain uint32_t* or a
// Strided view: word i of a lane at base[off + 32 * i], the per-lane tables
// of a warp interleaved in shared memory (bank = lane for every access).
// Offsets are 32-bit so address arithmetic stays in 32-bit registers.
struct Strided {
  uint32_t *base;
  int off;
  SARU_HD uint32_t &operator[](int i) const { return base[off + 32 * i]; }
  SARU_HD Strided operator+(int i) const { return Strided{base, off + 32 * i}; }
};

// bits [j, j + BITS) of a packed mask (words of 32 bits)
template <typename T, class P>
struct WindowBits;

template <class P>
struct WindowBits<uint32_t, P> {
  static SARU_HD uint32_t get(P mask, int j) {
    int w = j >> 5;
    return fshr32(mask[w], mask[w + 1], (uint32_t)j & 31u);
  }
};

template <class P>
struct WindowBits<uint64_t, P> {
  static SARU_HD uint64_t get(P mask, int j) {
    int w = j >> 5;
    uint32_t s = (uint32_t)j & 31u;
    uint32_t a = mask[w], b = mask[w + 1], c = mask[w + 2];
    uint32_t lo = fshr32(a, b, s);
    uint32_t hi = fshr32(b, c, s);
    return (uint64_t)lo | ((uint64_t)hi << 32);
  }
};

template <typename T, class P>
SARU_HD T window_bits(P mask, int j) {
  return WindowBits<T, P>::get(mask, j);
}

// bits [s, s + BITS) of the words at p (0 <= s < 32)
template <typename T, class P>
SARU_HD T window_bits_at(P p, int s);

template <>
SARU_HD uint32_t window_bits_at<uint32_t, Strided>(Strided p, int s) {
  return fshr32(p[0], p[1], (uint32_t)s);
}
template <>
SARU_HD uint64_t window_bits_at<uint64_t, Strided>(Strided p, int s) {
  const uint32_t a = p[0], b = p[1], c = p[2];
  return (uint64_t)fshr32(a, b, (uint32_t)s) | ((uint64_t)fshr32(b, c, (uint32_t)s) << 32);
}
template <>
SARU_HD uint32_t window_bits_at<uint32_t, uint32_t *>(uint32_t *p, int s) {
  return fshr32(p[0], p[1], (uint32_t)s);
}
template <>
SARU_HD uint64_t window_bits_at<uint64_t, uint32_t *>(uint32_t *p, int s) {
  const uint32_t a = p[0], b = p[1], c = p[2];
  return (uint64_t)fshr32(a, b, (uint32_t)s) | ((uint64_t)fshr32(b, c, (uint32_t)s) << 32);
}

SARU_HD int base_code(uint8_t c) {
  switch (c) {
    case 'A': return 0;
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    default: return -1;
  }
}

// Number of 32-bit mask words per read class for a window of length L.
SARU_HD int mask_words(int k, int L) { return ((k + 1 + L + 64) >> 5) + 1; }

// Per-candidate scalar description.
struct Cand {
  int m, L, k, so, eo;
  bool first_of_call;  // candidate 0 of a reference call: traceback stops on row 0
};

// Flags 1/5: end gap free (eo = k); 2/6: start gap (so = k); 3/7: both;
// anything else (0/4 are perfect hits): none.  Branch-free: bit 0 of a flag
// in 0..7 is the end gap, bit 1 the start gap.
SARU_HD void flank_of(int dir, int k, int &so, int &eo) {
  const bool valid = (unsigned)dir <= 7u;
  so = (valid && (dir & 2)) ? k : 0;
  eo = (valid && (dir & 1)) ? k : 0;
}

// Builds the read-class codes (4 bits each, 8 per word) and the window
// masks: bit (p + k + 1) of mask[c] is set iff window byte p belongs to
// class c.  Returns false if the read has more than MAX_EXTRA distinct
// non-ACGT bytes.  Reader/Writer abstract where bytes and words live.
template <class ReadFn, class WinFn, class P>
SARU_HD bool build_codes(const Cand &c, ReadFn rd, WinFn wn, P codes, P mask, int mwords) {
  uint8_t extra[MAX_EXTRA];
  int nextra = 0;
  for (int w = 0; w <= c.m / 8; ++w) codes[w] = 0;
  for (int j = 0; j < c.m; ++j) {
    uint8_t ch = rd(j);
    int code = base_code(ch);
    if (code < 0) {
      int e = 0;
      while (e < nextra && extra[e] != ch) ++e;
      if (e == nextra) {
        if (nextra == MAX_EXTRA) return false;
        extra[nextra++] = ch;
      }
      code = 4 + e;
    }
    codes[(j + 1) >> 3] |= (uint32_t)code << (((j + 1) & 7) * 4);
  }
  for (int w = 0; w < NCODES * mwords; ++w) mask[w] = 0;
  for (int p = 0; p < c.L; ++p) {
    uint8_t ch = wn(p);
    int code = base_code(ch);
    if (code < 0) {
      code = -1;
      for (int e = 0; e < nextra; ++e)
        if (extra[e] == ch) code = 4 + e;
      if (code < 0) continue;
    }
    int bit = p + c.k + 1;
    mask[code * mwords + (bit >> 5)] |= 1u << (bit & 31);
  }
  return true;
}

SARU_HD uint32_t byte_perm(uint32_t x, uint32_t y, uint32_t sel) {
#if defined(__CUDA_ARCH__)
  return __byte_perm(x, y, sel);
#else
  uint64_t v = (uint64_t)x | ((uint64_t)y << 32);
  uint32_t r = 0;
  for (int i = 0; i < 4; ++i) {
    uint32_t s = (sel >> (4 * i)) & 7u;
    r |= (uint32_t)((v >> (8 * s)) & 0xFFu) << (8 * i);
  }
  return r;
#endif
}

// Four bytes of ASCII -> their base codes (A=0 C=1 G=2 T=3 in the low two
// bits of each byte) and the ASCII those codes stand for; a byte is a base
// exactly when it equals that ASCII.
SARU_HD uint32_t base_codes4(uint32_t x) { return ((x >> 1) ^ (x >> 2)) & 0x03030303u; }
SARU_HD uint32_t codes4_nibbles(uint32_t c4) { return byte_perm(c4 | (c4 >> 4), 0, 0x4420); }
SARU_HD uint32_t ascii_of_nibbles(uint32_t nib) { return byte_perm(0x54474341u, 0, nib); }

// Fast build of the codes and masks when the read and the window hold only
// A/C/G/T (the common case).  rd4(i) / wn4(i) return bytes i..i+3 of the
// read / window, little endian; bytes past the sequence may be anything.
// Returns false (nothing guaranteed written) if a byte is not A/C/G/T.
template <class Rd4, class Wn4, class P>
SARU_HD bool build_codes_acgt(const Cand &c, Rd4 rd4, Wn4 wn4, P codes, P mask, int mwords) {
  uint32_t bad = 0;
  uint32_t prev = 0;  // the previous word's codes (its last nibble moves to the next word)
  for (int w = 0; 8 * w < c.m; ++w) {
    const uint32_t x0 = rd4(8 * w), x1 = rd4(8 * w + 4);
    const uint32_t s0 = codes4_nibbles(base_codes4(x0));
    const uint32_t s1 = codes4_nibbles(base_codes4(x1));
    const int left = c.m - 8 * w;  // chars of this word inside the read
    const uint32_t k0 = left >= 4 ? 0xFFFFFFFFu : ((1u << (8 * left)) - 1u);
    const uint32_t k1 = left >= 8 ? 0xFFFFFFFFu : (left > 4 ? ((1u << (8 * (left - 4))) - 1u) : 0u);
    bad |= ((ascii_of_nibbles(s0) ^ x0) & k0) | ((ascii_of_nibbles(s1) ^ x1) & k1);
    const uint32_t cw = s0 | (s1 << 16);
    codes[w] = (cw << 4) | (prev >> 28);
    prev = cw;
  }
  if (c.m % 8 == 0) codes[c.m / 8] = prev >> 28;
  if (bad) return false;
  // window bit-planes P0/P1 (code bits) over positions, 32 per word; mask
  // bit (p + k + 1) of class c is set iff window byte p is base c
  const int sh = c.k + 1;
  uint32_t prevA = 0, prevC = 0, prevG = 0, prevT = 0;
  const int words = (c.L + 31) >> 5;
  for (int q = 0; q < mwords; ++q) {
    uint32_t A = 0, C = 0, G = 0, T = 0;
    if (q < words) {
      uint32_t P0 = 0, P1 = 0;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const uint32_t x = wn4(32 * q + 4 * i);
        const uint32_t c4 = base_codes4(x);
        const int left = c.L - (32 * q + 4 * i);
        const uint32_t keep =
            left >= 4 ? 0xFFFFFFFFu : (left > 0 ? ((1u << (8 * left)) - 1u) : 0u);
        bad |= (ascii_of_nibbles(codes4_nibbles(c4)) ^ x) & keep;
        // bit 0 of each byte to bits 0..3, bit 1 to bits 4..7
        const uint32_t t = (c4 & 0x01010101u) | ((c4 << 3) & 0x10101010u);
        const uint32_t g = (t * 0x01020408u) >> 24;
        P0 |= (g & 0xFu) << (4 * i);
        P1 |= (g >> 4) << (4 * i);
      }
      const int inw = c.L - 32 * q;
      const uint32_t V = inw >= 32 ? 0xFFFFFFFFu : ((1u << inw) - 1u);
      A = ~P0 & ~P1 & V;
      C = P0 & ~P1 & V;
      G = ~P0 & P1 & V;
      T = P0 & P1 & V;
    }
    // shift the planes up by k+1 bits into mask word q (and carry)
    mask[0 * mwords + q] = sh >= 32 ? prevA : (A << sh) | (sh ? prevA >> (32 - sh) : 0u);
    mask[1 * mwords + q] = sh >= 32 ? prevC : (C << sh) | (sh ? prevC >> (32 - sh) : 0u);
    mask[2 * mwords + q] = sh >= 32 ? prevG : (G << sh) | (sh ? prevG >> (32 - sh) : 0u);
    mask[3 * mwords + q] = sh >= 32 ? prevT : (T << sh) | (sh ? prevT >> (32 - sh) : 0u);
    prevA = A;
    prevC = C;
    prevG = G;
    prevT = T;
  }
  return bad == 0;
}

template <class P>
SARU_HD int code_at(P codes, int j) {
  return (codes[(j + 1) >> 3] >> (((j + 1) & 7) * 4)) & 15;
}

// x >> 1 with the top bit set (one funnel shift a 32-bit word).
template <typename T>
SARU_HD T shr1_top(T x);
template <>
SARU_HD uint32_t shr1_top<uint32_t>(uint32_t x) {
  return fshr32(x, 1u, 1);
}
template <>
SARU_HD uint64_t shr1_top<uint64_t>(uint64_t x) {
  return (uint64_t)fshr32((uint32_t)x, (uint32_t)(x >> 32), 1) |
         ((uint64_t)fshr32((uint32_t)(x >> 32), 1u, 1) << 32);
}

// One column of the bit-parallel recurrence.  In: the previous column's
// vertical-delta vectors realigned to this column's rows (pv, mv) and the
// match vector eq.  Out: this column's vectors (Pv, Mv), the diagonal-zero
// vector d0 and the horizontal +1 vector hp.
template <typename T>
SARU_HD void myers_step(T pv, T mv, T eq, T &Pv, T &Mv, T &d0, T &hp) {
  const T xh = (((eq & pv) + pv) ^ pv) | eq;
  d0 = xh | mv;
  hp = mv | ~(d0 | pv);
  const T hn = pv & d0;
  const T hp1 = (hp << 1) | T(1);
  const T hn1 = hn << 1;
  Pv = hn1 | ~(d0 | hp1);
  Mv = hp1 & d0;
}

// Fill of one candidate.  `planes(j, A, B, last)` receives the decision planes of
// read column j (1..m): code = A | 2B per band bit.  Returns D[L][m] if it
// is <= k, otherwise k + 1.
template <typename T, class P, class PlaneSink>
SARU_HD int fill_band(const Cand &c, P codes, P mask, int mwords, PlaneSink planes) {
  constexpr int BITS = int(sizeof(T) * 8);
  const int k = c.k, m = c.m;
  const T TOPBIT = T(1) << (BITS - 1);
  // column 0: rows b - k; dv = -1 for rows <= 0, 0 for rows 1..2so, +1 after
  T Mv = lowmask<T>(k + 1);
  T Pv = ~lowmask<T>(k + 2 * c.so + 1);
  int top = k;  // D[j - k][j] for the current column j (virtual rows: j + (k - j))
  {
    // column 1, with the first-column quirk of the traceback: rows <= 2so+3
    // (bits <= 2so + k + 2) take the vertical test with cost 0
    const T eq = window_bits<T>(mask + (int)((codes[0] >> 4) & 15u) * mwords, 1);
    T d0, hp;
    myers_step<T>((Pv >> 1) | TOPBIT, Mv >> 1, eq, Pv, Mv, d0, hp);
    const T col1_corr = c.so ? lowmask<T>(2 * c.so + k + 3) : T(0);
    const T up = (Pv & ~col1_corr) | (~(Pv | Mv) & col1_corr);
    const T diag = ~d0 | eq;
    planes(1, diag | (~up & hp), ~diag & (up | hp), false);
    top += (int)((~d0) & T(1));
  }
  // columns 2..m-1; column j matches read byte j-1, nibble j & 7 of code
  // word j >> 3; the eight columns of a code word read mask words j >> 5
  // and (j >> 5) + 1 of the read byte's class
  for (int w = 0; 8 * w < m; ++w) {
    const uint32_t cw = codes[w];
    const P row = mask + (w >> 2);
    const int sh0 = 8 * (w & 3);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int j = 8 * w + i;
      if (j < 2) continue;
      if (j >= m) break;
      const int code = (int)((cw >> (4 * i)) & 15u);
      const T eq = window_bits_at<T>(row + code * mwords, sh0 + i);
      T d0, hp;
      myers_step<T>(shr1_top<T>(Pv), Mv >> 1, eq, Pv, Mv, d0, hp);
      const T diag = ~d0 | eq;
      planes(j, diag | (~Pv & hp), ~diag & (Pv | hp), false);
      top += (int)((~d0) & T(1));
    }
  }
  // column m with explicit values; column m-1 band values from the deltas
  const T eqm = window_bits<T>(mask + code_at(codes, m - 1) * mwords, m);
  const int bmax = c.L - m + k;  // band bit of row L in column m
  T A = 0, B = 0;
  int vb = top;           // D[m-1-k+b][m-1]: column m-1 at band bit b
  int vcur_prev = top + 1;  // D[m-k-1][m], entering from the left
  int score = k + 1;
  for (int b = 0; b <= bmax && b < BITS; ++b) {
    const int vb1 = b + 1 < BITS ? vb + (int)((Pv >> (b + 1)) & T(1)) - (int)((Mv >> (b + 1)) & T(1))
                                 : vb + 1;
    const int row = m - k + b;
    const int dg = vb, lf = vb1, tp = vcur_prev;
    const bool e = (eqm >> b) & T(1);
    const int corr = (row - 1 >= c.L - 2 * c.eo) ? 1 : 0;
    int v = dg + (e ? 0 : 1);
    if (lf + 1 < v) v = lf + 1;
    if (tp + 1 - corr < v) v = tp + 1 - corr;
    int op;
    if (dg + 1 == v || (dg == v && e)) op = OP_DIAG;
    else if (tp + 1 - corr == v) op = OP_UP;
    else if (lf + 1 == v) op = OP_LEFT;
    else op = OP_STOP;
    A |= T(op & 1) << b;
    B |= T(op >> 1) << b;
    vcur_prev = v;
    vb = vb1;
    if (b == bmax) score = v;
  }
  planes(m, A, B, true);
  return score <= k ? score : k + 1;
}

// Traceback from (L, m).  plane(j, b) returns the 2-bit decision of band bit
// b in column j.  emit(op, row, col) is called per step in traceback order
// (from the alignment end) with the cell the step leaves.  Returns the
// number of steps.
template <class PlaneFn, class EmitFn>
SARU_HD int traceback_band(const Cand &c, PlaneFn plane, EmitFn emit) {
  int row = c.L, col = c.m, n = 0;
  for (;;) {
    int op;
    if (col == 0) {
      // column 0 holds max(0, row - 2so); only the vertical test can hold
      if (row == 0) break;
      const int v = row - 2 * c.so > 0 ? row - 2 * c.so : 0;
      const int tp = row - 1 - 2 * c.so > 0 ? row - 1 - 2 * c.so : 0;
      const int corr = (c.so && row - 1 <= 2 * c.so + 2) ? 1 : 0;
      op = (tp + 1 - corr == v) ? OP_UP : OP_STOP;
    } else if (row == 0) {
      // row 0 holds j.  The first candidate of a call leaves the loop here;
      // the others see the previous matrix's last row as their diagonal and
      // top neighbours, all > k when m > 3k, so only the left step holds.
      op = c.first_of_call ? OP_STOP : OP_LEFT;
    } else {
      op = plane(col, row - col + c.k);
    }
    if (op == OP_STOP) break;
    emit(op, row, col);
    ++n;
    if (op == OP_DIAG) {
      --row;
      --col;
    } else if (op == OP_UP) {
      --row;
    } else {
      --col;
    }
  }
  return n;
}

}  // namespace saru

namespace saru {

// Maximum traceback length for a candidate: every step consumes a row or a
// column, and a path of value <= k makes at most k left steps.
SARU_HD int max_steps(const Cand &c) { return c.L + c.k; }

// Writes the reference's slot bytes for one traceback: ops[0..n) in
// traceback order (2 bits each, 16 per word), replayed from the cell where
// the traceback stopped so the strings come out in reading order, as the
// reference's in-place reversal leaves them (src/cuda-functions.cu:306-307).
template <class ReadFn, class WinFn, class OutFn>
SARU_HD void emit_forward(const Cand &c, const uint32_t *ops, int n, ReadFn rd, WinFn wn,
                          OutFn out) {
  int row = c.L, col = c.m;
  for (int s = 0; s < n; ++s) {
    int op = (ops[s >> 4] >> ((s & 15) * 2)) & 3;
    if (op == OP_DIAG) { --row; --col; }
    else if (op == OP_UP) { --row; }
    else { --col; }
  }
  // (row, col) is now the cell after the last step; walk back up the path
  for (int s = n - 1; s >= 0; --s) {
    int op = (ops[s >> 4] >> ((s & 15) * 2)) & 3;
    int r0 = row, c0 = col;
    if (op == OP_DIAG) { r0 = row + 1; c0 = col + 1; }
    else if (op == OP_UP) { r0 = row + 1; }
    else { c0 = col + 1; }
    uint8_t a = op == OP_UP ? (uint8_t)'_' : rd(c0 - 1);
    uint8_t b = op == OP_LEFT ? (uint8_t)'_' : wn(r0 - 1);
    out(n - 1 - s, a, b);
    row = r0;
    col = c0;
  }
}

}  // namespace saru
