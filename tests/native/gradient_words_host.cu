// Host build of the gradient kernel's per-pixel and per-index functions
// (dmsc_b200/csrc/gradient.cuh: gradient_tables, star_word, gather_offset,
// gather_index, crit_bits), for the CPU tests: the same code the device tiles run,
// applied to a whole image in plain loops, so the word encoding and the
// gather can be checked against the oracle without a GPU.
#include <cstdint>
#include <vector>

#include "../../dmsc_b200/csrc/gradient.cuh"

using namespace dmsc;

template <bool DUAL>
static void run(const float* img, int H, int W, int32_t* grad, uint8_t* mask, uint8_t* flow) {
  std::vector<uint32_t> lut(kGradTable);
  gradient_tables(lut.data());
  const int Nx = W + 1;
  // words of pixel (y, x) at [(y + 1) * (W + 2) + x + 1]; the border ring stays 0
  std::vector<uint32_t> w((size_t)(H + 2) * (W + 2), 0u);
  auto val = [&](int y, int x) { return (y >= 0 && y < H && x >= 0 && x < W) ? img[(size_t)y * W + x] : 0.0f; };
  // pixels with all eight neighbours take the 14-comparison table path (the
  // one interior device tiles run), the others the general path
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const bool inner = x >= 1 && x + 1 < W && y >= 1 && y + 1 < H;
      const float UL = val(y - 1, x - 1), U = val(y - 1, x), UR = val(y - 1, x + 1), L = val(y, x - 1),
                  P = val(y, x), R = val(y, x + 1), DL = val(y + 1, x - 1), D = val(y + 1, x), DR = val(y + 1, x + 1);
      w[(size_t)(y + 1) * (W + 2) + x + 1] =
          inner ? star_word<DUAL, true>(UL, U, UR, L, P, R, DL, D, DR, true, true, true, true, lut.data())
                : star_word<DUAL, false>(UL, U, UR, L, P, R, DL, D, DR, x >= 1, x + 1 < W, y >= 1, y + 1 < H,
                                         lut.data());
    }
  int off[32];
  for (int k = 0; k < 32; ++k) off[k] = gather_offset(k, Nx);
  for (int iy = 0; iy <= H; ++iy)
    for (int ix = 0; ix <= W; ++ix) {
      auto W_ = [&](int y, int x) { return w[(size_t)(y + 1) * (W + 2) + x + 1]; };
      const int b = iy * Nx + ix;
      int4 g;
      unsigned m, fl;
      gather_index(W_(iy, ix), W_(iy, ix - 1), W_(iy - 1, ix), W_(iy - 1, ix - 1), 4 * b, off, iy < H && ix < W, g,
                   m, fl);
      grad[4 * (size_t)b] = g.x;
      grad[4 * (size_t)b + 1] = g.y;
      grad[4 * (size_t)b + 2] = g.z;
      grad[4 * (size_t)b + 3] = g.w;
      // the compaction reads these bits back from the flow byte: both forms must agree
      const unsigned mb = crit_bits(fl, iy < H && ix < W);
      mask[b] = (uint8_t)(mb == m ? mb : 0xFFu);
      flow[b] = (uint8_t)fl;
    }
}

extern "C" void gradient_words_host(const float* img, int H, int W, int dual, int32_t* grad, uint8_t* mask,
                                    uint8_t* flow) {
  if (dual)
    run<true>(img, H, W, grad, mask, flow);
  else
    run<false>(img, H, W, grad, mask, flow);
}
