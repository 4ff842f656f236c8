// Pass plan of the pencil FFT passes (fft_pencil.cuh), shared by the host
// planner and the kernels of fft.cu.
#pragma once

#include <cstdint>

namespace dnufft {

constexpr int PEN_MAXL = 4;

struct PencilPlan {
  int L;                    // passes (0: no plan, radix-by-radix stages instead)
  int n;                    // line length
  int R[PEN_MAXL];          // radix of each pass
  int m[PEN_MAXL];          // stride of each pass: n / (R_1 ... R_i)
  int P[PEN_MAXL];          // twiddle index step: R_1 ... R_{i-1}
  uint32_t mmul[PEN_MAXL];  // ceil(2^32 / m_i): pencil -> (segment, offset) without division
};

}  // namespace dnufft
