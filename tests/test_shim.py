"""The reference-side binding (cfd-simulator_b200/shim/gpu_simple_solver.hpp):
the reference's SimpleSolver interface over the C ABI, for SolverWorker,
updateSolver and the tests' converge() loops.

On CPU: the header compiles against the reference's own headers with
warnings as errors (where the reference's headers are present). On a GPU:
oracle/shim_check (built next to the reference by `make -C oracle shim`)
drives it as the reference's callers do, beside the reference's solver on the
same mesh, and checks the converged fields (1e-9 relative L2), the turbulence
model's fields and y+, and Cl/Cd/Cm from the reference's own extractSurface
and integrateForces (1e-7 relative), plus move-only ownership, the error-code
mapping and the mutable field() round trip."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "cfd-simulator_b200", "shim")
DRIVER = os.path.join(ROOT, "oracle", "_ref", "shim_check")


def _reference_include():
    """The reference checkout's include directory, from the oracle recipe's REF."""
    try:
        path = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                              capture_output=True, text=True, check=True).stdout.strip()
    except (OSError, subprocess.CalledProcessError):
        return None
    if not path:
        return None
    inc = os.path.join(path, "include")
    return inc if os.path.isdir(os.path.join(inc, "cfd", "solver")) else None


def test_binding_compiles_against_the_reference_headers(tmp_path):
    inc = _reference_include()
    if inc is None:
        pytest.skip("the reference's headers are not present on this machine")
    src = tmp_path / "use.cpp"
    src.write_text(
        '#include "gpu_simple_solver.hpp"\n'
        "#include <optional>\n"
        "// SolverWorker holds its solver as std::optional<SimpleSolver> and moves one in\n"
        "void adopt(std::optional<cfd::solver::gpu::GpuSimpleSolver>& slot,\n"
        "           cfd::solver::gpu::GpuSimpleSolver s) { slot.emplace(std::move(s)); }\n"
        "static_assert(!std::is_copy_constructible_v<cfd::solver::gpu::GpuSimpleSolver>);\n"
        "static_assert(std::is_nothrow_move_constructible_v<cfd::solver::gpu::GpuSimpleSolver>);\n")
    out = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
                          f"-I{inc}", f"-I{os.path.join(ROOT, 'include')}", f"-I{SHIM}", str(src)],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


@pytest.mark.gpu
def test_binding_drives_the_device_like_the_reference_solver():
    if not os.path.exists(DRIVER):
        pytest.fail(f"{DRIVER} is missing: build it with `make -C oracle shim` where the "
                    "reference sources are present")
    out = subprocess.run([DRIVER], capture_output=True, text=True, timeout=900)
    lines = out.stdout.splitlines()
    failed = [ln for ln in lines if ln.startswith("check ") and ln.endswith("FAILED")]
    assert out.returncode == 0 and not failed, "\n".join(lines[-40:]) + out.stderr[-2000:]
    checks = {ln.split()[1] for ln in lines if ln.startswith("check ")}
    for name in ("short_conditions", "relaxation_refused", "unsupported_model", "move_leaves_no_handle",
                 "fields_1e-9", "turbulence_fields_1e-9", "yplus", "forces_1e-7",
                 "mutable_field_roundtrip_exact"):
        assert name in checks, name
