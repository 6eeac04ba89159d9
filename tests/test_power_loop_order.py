"""The power loop's step order on the CPU, with no device: the library's own
run_power_loop (scx_b200/csrc/power_loop.h, which the plan drives on the GPU)
instantiated over a recording and a symbolic fake (tests/cpp/power_loop_fakes.cpp),
as the reference pins run_power_loop with its RecordingOperator and
SymbolicOperator (scx-gpu/src/pca_operator_tests.rs:32-126): the exact sequence
for each iteration count, 4 + 4N steps (the reference's 3 + 4N plus the explicit
formation of Q that the implicit-Q loop needs), a failing step ends the loop
there, and each product reads the buffer it should."""

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "power_loop_fakes.cpp"


@pytest.fixture(scope="module")
def fakes(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = tmp_path_factory.mktemp("fakes") / "power_loop_fakes"
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", str(ROOT / "scx_b200" / "csrc"), str(SRC), "-o", str(out)],
                   check=True)
    return out


def _run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, check=True)
    return r.stdout.split()


def expected(n):
    want = ["matmat(Omega,last)" if n == 0 else "matmat(Omega)", "qr(Y)"]
    for it in range(n):
        want += ["rmatmat", "qr(Z)", "matmat(Z,last)" if it == n - 1 else "matmat(Z)", "qr(Y)"]
    return want + ["finalize_q", "rmatmat"]


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4])
def test_sequence_for_each_iteration_count(fakes, n):
    out = _run(fakes, "record", n)
    assert out[-1] == "OK"
    assert out[:-1] == expected(n)
    assert len(out) - 1 == 4 + 4 * n


def test_zero_iterations_still_seed_factor_and_project(fakes):
    assert _run(fakes, "record", 0)[:-1] == ["matmat(Omega,last)", "qr(Y)", "finalize_q", "rmatmat"]


@pytest.mark.parametrize("fail_at", [0, 1, 2, 5, 9])
def test_a_failing_step_ends_the_loop_there(fakes, fail_at):
    out = _run(fakes, "record", 2, fail_at)
    assert out[-1] == "FAILED"
    assert out[:-1] == expected(2)[: fail_at + 1]


def test_each_step_reads_the_right_buffer(fakes):
    y, z = _run(fakes, "symbolic", 2)
    q1 = "q(X.W)"
    q2 = f"q(X.q(Xt.{q1}))"
    q3 = f"q(X.q(Xt.{q2}))"
    assert y == f"Y={q3}"
    assert z == f"Z=Xt.{q3}"
