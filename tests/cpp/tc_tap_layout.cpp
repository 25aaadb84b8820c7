// Host check of the tensor-core filtering's packed taps (no GPU needed).
//
// The kernel multiplies, for every (input-plane offset c, dy) stage, a
// 128 x 16 banded Toeplitz matrix A by the staged input samples.  Row
// r = (stacked plane s, real filter f, x offset xo) holds the 7 taps
// F_f[3 - dz][3 - dy][3 - dx] (dz = c - s) at samples xo .. xo + 6.  This
// program rebuilds A from what the library packs and compares it with that
// definition:
//   split BF16: A = hi + lo, two K-major blocks of 8 samples per part, to
//     within 2^-16 of the FP32 tap;
//   TF32: one stored value per sample pair (P, P + 8), the kept sample named
//     by the metadata nibble (0b0100 the first, 0b1110 the second) that the
//     kernel writes to TMEM lane m0 + 8 k1 + 16 m2 for rows m0 + 8 m1 + 16 m2
//     (bits 16 m1 + 4 j, pair P = 4 k1 + j); bit-exact against the tap
//     rounded to TF32 (nearest, ties away from zero).
// Prints "ok" and exits 0, or names the first mismatch and exits 1.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

namespace brc {
namespace tc {
size_t packed_tap_bytes(int nfilt, bool tf32);
void pack_taps(const float* h_filters, int nfilt, uint16_t* dst, bool tf32);
uint32_t metadata_word(int lane, int SP, int nfilt);
}  // namespace tc
}  // namespace brc

namespace {

constexpr int kM = 128, kXo = 10, kTaps = 343, kFilterFloats = 686;

float bits_to_float(uint32_t b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

uint32_t tf32_bits(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  if ((b & 0x7f800000u) == 0x7f800000u) return b;  // inf / nan unchanged
  return (b + 0x1000u) & 0xffffe000u;             // 13 dropped bits, ties away
}

// The dense A row of stage (cq, dyq), row r: the tap at each of 16 samples
// (0 where the row has none).
void dense_row(const std::vector<float>& bank, int nfilt, int cq, int dyq, int r, float* row) {
  for (int k = 0; k < 16; k++) row[k] = 0.f;
  const int SP = nfilt == 3 ? 2 : 1;
  int s = 0, rr = r;
  if (SP == 2) {
    s = r >> 6;
    rr = r & 63;
  }
  if (rr >= 2 * nfilt * kXo) return;
  const int f = rr / kXo, xo = rr % kXo;
  const int dz = (cq - 3) - s, dy = dyq - 3;
  if (dz < -3 || dz > 3) return;
  const float* F = bank.data() + (size_t)(f >> 1) * kFilterFloats + (f & 1) * kTaps;
  for (int kx = xo; kx <= xo + 6; kx++) {
    const int dx = kx - 3 - xo;
    row[kx] = F[(3 - dz) * 49 + (3 - dy) * 7 + (3 - dx)];
  }
}

int check(int nfilt, bool tf32, unsigned seed) {
  std::mt19937 gen(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> bank((size_t)nfilt * kFilterFloats);
  for (auto& v : bank) v = nd(gen) * 0.05f;
  const size_t bytes = brc::tc::packed_tap_bytes(nfilt, tf32);
  std::vector<uint16_t> packed(bytes / 2);
  brc::tc::pack_taps(bank.data(), nfilt, packed.data(), tf32);
  const int SP = nfilt == 3 ? 2 : 1;
  const size_t stage_halves = tf32 ? (size_t)kM * 8 * 2 : (size_t)kM * 16 * 2;
  if (bytes != (size_t)28 * 2 * stage_halves * 2) {
    std::fprintf(stderr, "nfilt %d tf32 %d: %zu packed bytes\n", nfilt, (int)tf32, bytes);
    return 1;
  }
  uint32_t meta[kM];
  for (int L = 0; L < kM; L++) meta[L] = brc::tc::metadata_word(L, SP, nfilt);
  int checked = 0;
  for (int cq = 0; cq < 8; cq++)
    for (int dyq = 0; dyq < 7; dyq++) {
      const size_t stage = (size_t)(dyq * 4 + cq / 2) * 2 + (cq & 1);
      const uint16_t* base = packed.data() + stage * stage_halves;
      const bool present = cq < 6 + SP;  // cq = 7 exists with two stacked planes only
      for (int r = 0; r < kM; r++) {
        float want[16];
        if (present)
          dense_row(bank, nfilt, cq, dyq, r, want);
        else
          for (int k = 0; k < 16; k++) want[k] = 0.f;
        float got[16];
        if (tf32) {
          for (int k = 0; k < 16; k++) got[k] = 0.f;
          const int m0 = r & 7, m1 = (r >> 3) & 1, m2 = r >> 4;
          for (int P = 0; P < 8; P++) {
            const size_t e = (size_t)(P / 4) * (kM * 4) + (size_t)r * 4 + (P % 4);
            uint32_t b;
            std::memcpy(&b, base + 2 * e, 4);
            const int L = m0 + 8 * (P >> 2) + 16 * m2;
            const uint32_t nib = (meta[L] >> (16 * m1 + 4 * (P & 3))) & 0xfu;
            if (nib != 0x4u && nib != 0xeu) {
              std::fprintf(stderr, "nfilt %d row %d pair %d: metadata nibble %x\n", nfilt, r, P, nib);
              return 1;
            }
            got[nib == 0x4u ? P : P + 8] = bits_to_float(b);
          }
          for (int k = 0; k < 16; k++) {
            const uint32_t wb = tf32_bits(want[k]);
            uint32_t gb;
            std::memcpy(&gb, &got[k], 4);
            if (gb != wb) {
              std::fprintf(stderr, "tf32 nfilt %d cq %d dyq %d row %d sample %d: %08x, want %08x\n", nfilt, cq,
                           dyq, r, k, gb, wb);
              return 1;
            }
          }
        } else {
          const uint16_t* hi = base;
          const uint16_t* lo = base + (size_t)kM * 16;
          for (int k = 0; k < 16; k++) {
            const size_t e = (size_t)(k / 8) * (kM * 8) + (size_t)r * 8 + (k % 8);
            got[k] = bits_to_float((uint32_t)hi[e] << 16) + bits_to_float((uint32_t)lo[e] << 16);
            if (std::fabs(got[k] - want[k]) > std::ldexp(std::fabs(want[k]), -16)) {
              std::fprintf(stderr, "bf16x3 nfilt %d cq %d dyq %d row %d sample %d: %g, want %g\n", nfilt, cq,
                           dyq, r, k, got[k], want[k]);
              return 1;
            }
          }
        }
        checked++;
      }
    }
  return checked == 8 * 7 * kM ? 0 : 1;
}

}  // namespace

int main() {
  int bad = 0;
  for (int nfilt : {3, 6})
    for (bool tf32 : {false, true}) bad |= check(nfilt, tf32, 17u * nfilt + (tf32 ? 1u : 0u));
  if (bad) return 1;
  std::printf("ok\n");
  return 0;
}
