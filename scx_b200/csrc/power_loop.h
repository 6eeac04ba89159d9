// The step order of the randomized power loop, written once and driven over
// any operator: the plan's device operator (scxpca.cu) and the recording and
// symbolic fakes of the CPU tests.  Restates run_power_loop
// (scx-gpu/src/pca_operator.rs:100-119):
//
//   matmat(Omega) -> qr(Y) -> [ rmatmat -> qr(Z) -> matmat(Z) -> qr(Y) ] x N
//     -> finalize_q -> rmatmat
//
// with one step the reference does not need: finalize_q.  The device
// operator keeps the Y factor implicit inside the loop (Q = Y R^-1 is folded
// into the next transposed product), so before the closing product it forms
// Q explicitly and re-orthonormalises it.  The closing rmatmat leaves
// B = (X - 1 mu^T)^T Q for the Rayleigh-Ritz step.  Operator failures are
// exceptions: a step that throws ends the loop there.
#pragma once

#include <cstdint>

namespace scx {

enum class Operand { kOmega, kZ };  // the right operand of a forward product
enum class Buf { kY, kZ };          // the buffer a factorisation orthonormalises

// Op provides:
//   void matmat(Operand src, bool last)  Y <- (X - 1 mu^T) src; `last` marks
//                                        the loop's final forward product
//   void rmatmat()                       Z <- (X - 1 mu^T)^T Q
//   void qr(Buf b)                       b <- an orthonormal basis of b
//   void finalize_q()                    the loop's Q made explicit and
//                                        re-orthonormalised
template <class Op>
void run_power_loop(Op& op, int64_t n_power_iterations) {
  op.matmat(Operand::kOmega, n_power_iterations == 0);
  op.qr(Buf::kY);
  for (int64_t it = 0; it < n_power_iterations; ++it) {
    op.rmatmat();
    op.qr(Buf::kZ);
    op.matmat(Operand::kZ, it + 1 == n_power_iterations);
    op.qr(Buf::kY);
  }
  op.finalize_q();
  op.rmatmat();
}

}  // namespace scx
