// CPU fakes of the power-loop operator, driven by the library's own
// run_power_loop (scx_b200/csrc/power_loop.h).  The counterpart of the
// reference's RecordingOperator and SymbolicOperator
// (scx-gpu/src/pca_operator_tests.rs:32-126): the recording fake prints the
// exact step sequence (and can fail at step n, which must end the loop
// there); the symbolic fake tracks what each buffer holds as an expression, so
// a step that reads the wrong buffer shows up even when the sequence is right.
//
// Usage: power_loop_fakes record <n_power_iterations> [fail_at]
//        power_loop_fakes symbolic <n_power_iterations>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "power_loop.h"

using scx::Buf;
using scx::Operand;

struct Recording {
  std::vector<std::string> steps;
  long fail_at = -1;
  void record(const std::string& s) {
    steps.push_back(s);
    if ((long)steps.size() - 1 == fail_at) throw std::runtime_error("fake failure at " + s);
  }
  void matmat(Operand src, bool last) {
    record(std::string("matmat(") + (src == Operand::kOmega ? "Omega" : "Z") + (last ? ",last)" : ")"));
  }
  void rmatmat() { record("rmatmat"); }
  void qr(Buf b) { record(b == Buf::kY ? "qr(Y)" : "qr(Z)"); }
  void finalize_q() { record("finalize_q"); }
};

struct Symbolic {
  std::string y = "?", z = "?";
  void matmat(Operand src, bool) { y = "X." + (src == Operand::kOmega ? std::string("W") : z); }
  void rmatmat() { z = "Xt." + y; }
  void qr(Buf b) {
    if (b == Buf::kY) y = "q(" + y + ")";
    else z = "q(" + z + ")";
  }
  void finalize_q() {}  // the same Q, made explicit: the buffer's content is unchanged
};

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const long q = std::atol(argv[2]);
  if (!std::strcmp(argv[1], "record")) {
    Recording op;
    if (argc > 3) op.fail_at = std::atol(argv[3]);
    bool failed = false;
    try {
      scx::run_power_loop(op, q);
    } catch (const std::exception&) {
      failed = true;
    }
    for (const auto& s : op.steps) std::printf("%s\n", s.c_str());
    std::printf(failed ? "FAILED\n" : "OK\n");
    return 0;
  }
  if (!std::strcmp(argv[1], "symbolic")) {
    Symbolic op;
    scx::run_power_loop(op, q);
    std::printf("Y=%s\nZ=%s\n", op.y.c_str(), op.z.c_str());
    return 0;
  }
  return 2;
}
