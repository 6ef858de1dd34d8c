// Shape and parameter layout of the learned smoother's MLP (29 -> 64 -> 64 -> 20).
//   W1 [64][29], b1 [64], W2 [64][64], b2 [64], W3 [20][64], b3 [20]
#pragma once

namespace sfem {

struct MLPDims {
  static constexpr int NIN = 29, NH = 64, NOUT = 20, NR = 20, NJ = 9;
  static constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NIN, OFF_W2 = OFF_B1 + NH;
  static constexpr int OFF_B2 = OFF_W2 + NH * NH, OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NOUT * NH;
  static constexpr int NPARAM = OFF_B3 + NOUT;  // 7380
};

}  // namespace sfem
