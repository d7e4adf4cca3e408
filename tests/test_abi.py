"""The C-ABI library loads, exports every entry point include/iblbm_b200.h
declares, and the ctypes structures match the C layout (CPU only: no kernel
is launched)."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "iblbm_b200.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^int\s+(iblbm_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from iblbm_b200 import _lib
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 10
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(_lib._SIGS), set(names) - set(_lib._SIGS)


def test_struct_layout_matches_c(tmp_path):
    from iblbm_b200 import _lib
    probe = tmp_path / "probe.c"
    fields = {"iblbm_ibm_args": [f for f, _ in _lib.IbmArgs._fields_],
              "iblbm_dense_args": [f for f, _ in _lib.DenseArgs._fields_],
              "iblbm_ibm32_args": [f for f, _ in _lib.Ibm32Args._fields_],
              "iblbm_dense32_args": [f for f, _ in _lib.Dense32Args._fields_],
              "iblbm_case": [f for f, _ in _lib.Case._fields_],
              "iblbm_force_coeff_args": [f for f, _ in _lib.ForceCoeffArgs._fields_],
              "iblbm_velocity_change_args": [f for f, _ in _lib.VelocityChangeArgs._fields_],
              "iblbm_particles_args": [f for f, _ in _lib.ParticlesArgs._fields_]}
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){"]
    for st, fl in fields.items():
        lines.append(f'printf("{st} %zu\\n", sizeof({st}));')
        for f in fl:
            cf = "lambda" if f == "lambda_" else f
            lines.append(f'printf("{st}.{f} %zu\\n", offsetof({st}, {cf}));')
    lines.append('printf("IBLBM_PARTICLE_STATE %d\\n", IBLBM_PARTICLE_STATE);')
    lines.append('printf("IBLBM_PARTICLE_CONSTS %d\\n", IBLBM_PARTICLE_CONSTS);')
    lines.append("return 0;}")
    probe.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.check_call(["gcc", str(probe), "-o", str(exe)])
    out = dict(l.rsplit(" ", 1) for l in subprocess.check_output([str(exe)]).decode().split("\n") if l)
    for st, cls in (("iblbm_ibm_args", _lib.IbmArgs), ("iblbm_dense_args", _lib.DenseArgs),
                    ("iblbm_ibm32_args", _lib.Ibm32Args), ("iblbm_dense32_args", _lib.Dense32Args),
                    ("iblbm_case", _lib.Case), ("iblbm_force_coeff_args", _lib.ForceCoeffArgs),
                    ("iblbm_velocity_change_args", _lib.VelocityChangeArgs),
                    ("iblbm_particles_args", _lib.ParticlesArgs)):
        assert int(out[st]) == ctypes.sizeof(cls), st
        for f, _ in cls._fields_:
            assert int(out[f"{st}.{f}"]) == getattr(cls, f).offset, (st, f)
    assert int(out["IBLBM_PARTICLE_STATE"]) == _lib.PARTICLE_STATE
    assert int(out["IBLBM_PARTICLE_CONSTS"]) == _lib.PARTICLE_CONSTS


def test_rejects_bad_arguments_without_a_gpu():
    """Argument validation happens on the host before any launch."""
    from iblbm_b200 import _lib
    L = _lib.lib()
    assert L.iblbm_dense_step_f64(None, None) == -1
    assert L.iblbm_ibm_step_f64(None, None) == -1
    assert L.iblbm_dense_step_f32(None, None) == -1
    assert L.iblbm_ibm_step_f32(None, None) == -1
    assert L.iblbm_feq(None, None, 10, 0, None, None) == -1


def test_particle_step_rejects_bad_arguments_without_a_gpu():
    """The particle step's phase and rotation checks run on the host before any
    launch (the pointers here are never dereferenced)."""
    import ctypes
    from iblbm_b200 import _lib
    L = _lib.lib()
    fake = ctypes.c_void_p(16)

    def args(**over):
        a = _lib.ParticlesArgs()
        a.n_particles, a.model, a.band_capacity, a.nx, a.ny, a.dy = 2, 0, 10, 10, 10, 1.0
        for f in ("moff", "state", "consts", "band_fib_part", "band_count", "Lx_c", "Ly_c", "Lx", "Ly", "dvel",
                  "band_nodes", "rho", "U", "lint_scratch"):
            setattr(a, f, fake)
        a.lint_capacity = 100
        for k, v in over.items():
            setattr(a, k, v)
        return a

    E_ARG = -1
    step = lambda a: L.iblbm_particles_step_f64(ctypes.byref(a), None)
    assert step(args(phase=0)) == E_ARG
    assert step(args(phase=4 | 1)) == E_ARG          # Euler is a whole step on its own
    assert step(args(phase=8)) == E_ARG
    assert step(args(phase=2, rotation=1, band_nodes=None)) == E_ARG
    assert step(args(phase=2, rotation=1, dy=0.0)) == E_ARG
    assert step(args(phase=4, rotation=1, rho=None)) == E_ARG
    assert step(args(phase=4, rotation=1, lint_capacity=0)) == E_ARG
    assert step(args(phase=4, rotation=1, lint_capacity=1 << 20)) == E_ARG
    assert step(args(phase=3, n_particles=9)) == E_ARG
    assert step(args(phase=3, lagrangian=3)) == E_ARG
    assert step(args(phase=3, lagrangian=1, Lfx=None)) == E_ARG     # DF sums need the marker forces
    assert step(args(phase=3, lagrangian=2, dfc_force=None)) == E_ARG
    assert step(args(phase=3, prescribed=1, rotation=1)) == E_ARG   # a prescribed disc does not turn
    assert step(args(phase=4, prescribed=1)) == E_ARG


def test_cluster_plan_sizes():
    """Which bodies the cluster form of the FP64 MDF step takes (no GPU needed)."""
    from iblbm_b200._lib import lib
    L = lib()
    assert L.iblbm_ibm_cluster_plan_ints(126, 0, 8) > 0
    assert L.iblbm_ibm_cluster_plan_ints(152, 0, 8) > 0
    assert L.iblbm_ibm_cluster_plan_ints(153, 0, 8) > 0
    assert L.iblbm_ibm_cluster_plan_ints(126, 0, 2) > 0
    assert L.iblbm_ibm_cluster_plan_ints(1025, 0, 8) == 0  # 129 markers per CTA: 5 marker warps x 8 > 32 slots
    assert L.iblbm_ibm_cluster_plan_ints(392, 1, 8) > 0
    assert L.iblbm_ibm_cluster_plan_ints(126, 0, 3) == 0
    assert L.iblbm_ibm_cluster_plan_ints(4, 1, 8) == 0
