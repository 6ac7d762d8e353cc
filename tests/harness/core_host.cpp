// Host build of the device alignment core (saruman_b200/csrc/saru_core.cuh)
// for CPU tests of the algorithm against the oracle.  Test infrastructure:
// the product runs the same header on the GPU only.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../saruman_b200/csrc/saru_core.cuh"

using namespace saru;

template <typename T>
static int run(const Cand &c, const uint8_t *read, const uint8_t *win, int *score, uint8_t *ra,
               uint8_t *ga) {
  const int mw = mask_words(c.k, c.L);
  std::vector<uint32_t> codes((c.m + 7) / 8 + 1), mask(NCODES * mw);
  // padded copies: the word readers look up to 40 bytes past the end
  std::vector<uint8_t> rpad(c.m + 64, 0xEE), wpad(c.L + 64, 0xEE);
  memcpy(rpad.data(), read, c.m);
  memcpy(wpad.data(), win, c.L);
  auto ld4 = [](const uint8_t *p) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
  };
  if (!build_codes_acgt(c, [&](int i) { return ld4(rpad.data() + i); },
                        [&](int i) { return ld4(wpad.data() + i); }, codes.data(), mask.data(),
                        mw) &&
      !build_codes(c, [&](int j) { return read[j]; }, [&](int p) { return win[p]; },
                   codes.data(), mask.data(), mw))
    return 1;
  std::vector<T> PA(c.m + 1), PB(c.m + 1);
  int s = fill_band<T>(c, codes.data(), mask.data(), mw, [&](int j, T A, T B, bool) {
    PA[j] = A;
    PB[j] = B;
  });
  *score = s;
  if (s > c.k) return 0;
  std::vector<uint32_t> ops((max_steps(c) + 15) / 16 + 1);
  int bad = 0;
  int n = traceback_band(
      c,
      [&](int j, int b) -> int {
        if (b < 0 || b >= int(sizeof(T) * 8)) {
          bad = 1;
          return OP_STOP;
        }
        return int((PA[j] >> b) & 1) | (int((PB[j] >> b) & 1) << 1);
      },
      [&](int op, int, int) {
        static_cast<void>(0);
        (void)op;
      });
  // second walk to collect ops (the kernel keeps them in registers/local)
  int idx = 0;
  std::fill(ops.begin(), ops.end(), 0u);
  traceback_band(
      c,
      [&](int j, int b) -> int {
        if (b < 0 || b >= int(sizeof(T) * 8)) return OP_STOP;
        return int((PA[j] >> b) & 1) | (int((PB[j] >> b) & 1) << 1);
      },
      [&](int op, int, int) {
        ops[idx >> 4] |= uint32_t(op) << ((idx & 15) * 2);
        ++idx;
      });
  if (n > max_steps(c)) return 2;
  emit_forward(c, ops.data(), n, [&](int j) { return read[j]; }, [&](int p) { return win[p]; },
               [&](int pos, uint8_t a, uint8_t b) {
                 ra[pos] = a;
                 ga[pos] = b;
               });
  return bad ? 3 : 0;
}

// Same call layout as the reference; returns a bitmask of per-candidate
// problems (1 = unsupported read alphabet, 2 = overlong, 3 = band escape).
extern "C" int core_align_batch(const uint8_t *genome, const uint8_t *reads, const int *goff,
                                const int *roff, const int8_t *dirs, int n, int k, int wide,
                                int first_of_call, int *scores, uint8_t *ra, uint8_t *ga) {
  int flags = 0;
  long slot = 0;
  for (int t = 0; t < n; ++t) {
    long gs = t ? goff[t - 1] : 0, rs = t ? roff[t - 1] : 0;
    Cand c;
    c.m = int(roff[t] - rs);
    c.L = int(goff[t] - gs);
    c.k = k;
    flank_of(dirs[t], k, c.so, c.eo);
    c.first_of_call = first_of_call && t == 0;
    int st = wide ? run<uint64_t>(c, reads + rs, genome + gs, &scores[t], ra + slot, ga + slot)
                  : run<uint32_t>(c, reads + rs, genome + gs, &scores[t], ra + slot, ga + slot);
    if (st) flags |= 1 << (st - 1);
    slot += c.L + k;
  }
  return flags;
}
