"""C-ABI checks that need no GPU: every function declared in include/hfb.h is
exported by libhfb.so and bound in hfb._lib; the ctypes structure layouts
match the C compiler's; host-side set-up logic matches the oracle."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "hfb.h")


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*|unsigned long long)\s+(hfb_\w+)\s*\(", txt, re.M)))


@pytest.fixture(scope="module")
def lib():
    from hfb import _lib
    if not os.path.exists(_lib.LIB_PATH):
        import build as b
        b.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    from hfb import _lib
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SYMBOLS)


def test_status_strings(lib):
    from hfb import _lib
    for code in range(8):
        assert lib.hfb_status_string(code).decode()
    assert lib.hfb_status_string(4).decode().startswith("BCS")


def test_ctx_create_rejects_bad_grids_without_gpu(lib):
    h = C.c_void_p()
    # non-cubic and odd grids are rejected before any device call
    assert lib.hfb_ctx_create(16, 16, 24, 1.0, 1.0, 1.0, 0, 0, C.byref(h)) == 2
    assert lib.hfb_ctx_create(15, 15, 15, 1.0, 1.0, 1.0, 0, 0, C.byref(h)) == 1
    assert lib.hfb_ctx_create(20, 20, 20, 1.0, 1.0, 1.0, 0, 0, C.byref(h)) == 2


def test_null_arguments_are_rejected(lib):
    assert lib.hfb_hpsi(None, 0, None, 1, 1, None, None, None, None, None, None, None) == 1
    assert lib.hfb_pair(None, None, None) == 1
    # observables, single-particle properties and constraints: a missing
    # context or buffer is HFB_ERR_ARG before any device work
    assert lib.hfb_observables(None, None, None, 8.0, 8.0, None, None) == 1
    assert lib.hfb_sp_properties(None, 0, 4, None, None, None, None, None, None) == 1
    assert lib.hfb_constraint_fields(None, 1, 16.0, 0.93, 6.0, 1.0, None, None) == 1
    assert lib.hfb_constraint_moments(None, 1, None, None, None, None) == 1
    assert lib.hfb_constraint_potential(None, 0, 1, None, None, None, None, None) == 1
    assert lib.hfb_constraint_correct(None, 0, 1, 1, None, None, None, None, None, None) == 1


def test_struct_layouts_match_c():
    """Compile a probe against include/hfb.h and compare sizeof / offsetof."""
    from hfb import _lib
    structs = {"hfb_force": _lib.HfbForce, "hfb_grstep_args": _lib.GrstepArgs, "hfb_diag_args": _lib.DiagArgs,
               "hfb_pair_args": _lib.PairArgs}
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = {}
    for ln in out.splitlines():
        s, f, v = ln.split()
        got[(s, f)] = int(v)
    for cname, cls in structs.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_ho_quantum_numbers_match_oracle():
    from hfb.static import ho_quantum_numbers
    from oracle.static import ho_quantum_numbers as ref
    for n in (1, 2, 10, 32, 96, 140):
        assert ho_quantum_numbers(n) == ref(n)


def test_force_coefficients_match_oracle():
    from hfb.forces import init_forces
    from oracle.model import init_forces as ref
    for ipair in (0, 5, 6):
        a = init_forces(None, name="SLy4", ipair=ipair)
        b = ref("SLy4", ipair=ipair)
        for k in ("b0", "b0p", "b1", "b1p", "b2", "b2p", "b3", "b3p", "b4", "b4p", "slate", "Crho0", "Crho1",
                  "Crho0D", "Crho1D", "Cdrho0", "Cdrho1", "Ctau0", "Ctau1", "CdJ0", "CdJ1", "h2ma", "v0prot",
                  "v0neut", "rho0pr"):
            assert getattr(a, k) == pytest.approx(getattr(b, k), rel=1e-15, abs=1e-15), k
        s = a.c_struct()
        assert s.b0 == a.b0 and s.ipair == ipair


def test_oscillator_radii():
    from hfb.config import ho_radii, case_dict
    rx, ry, rz = ho_radii(8, 8)
    assert rx == ry == rz
    assert abs(rx - 2.2576) < 1e-3      # radin = sqrt(2) b, b^2 = 2 h2m / (41 A^-1/3)
    rx, ry, rz = ho_radii(24, 24, beta=0.2)
    assert rz > rx and abs(rx * ry * rz - ho_radii(24, 24)[0] ** 3) < 1e-9
    c = case_dict("Pb208")
    assert c["levels"]["npsi"] == [140, 96] and c["grid"]["nx"] == 48


def test_force_jacobian_matches_finite_differences():
    """db/dtheta used by the energy sensitivities equals finite differences
    of the coefficient formulas of init_forces."""
    from hfb import adjoint
    from hfb.forces import init_forces
    base = init_forces(None, name="SLy4", ipair=5)
    jac = adjoint._db_dtheta(base)
    th0 = adjoint.theta_of(base)
    for name, row in jac.items():
        h = 1e-6 * abs(th0[name])
        fp = init_forces(None, name="SLy4", ipair=5,
                         overrides=adjoint.force_overrides(dict(force=dict(name="SLy4")),
                                                           {name: th0[name] + h})["force"]["overrides"])
        fm = init_forces(None, name="SLy4", ipair=5,
                         overrides=adjoint.force_overrides(dict(force=dict(name="SLy4")),
                                                           {name: th0[name] - h})["force"]["overrides"])
        for b in ("b0", "b0p", "b1", "b1p", "b2", "b2p", "b3", "b3p", "b4", "b4p"):
            d = (getattr(fp, b) - getattr(fm, b)) / (2 * h)
            assert d == pytest.approx(row.get(b, 0.0), rel=1e-6, abs=1e-9), (name, b)


def test_res_writer_matches_reference_text(tmp_path):
    """hfb.output.FortranOutputWriter writes the same bytes as the
    reference's writer (output.py:49-174) for the seeded inputs of
    tests/golden/res_files.json."""
    import json
    import types
    import numpy as np
    from hfb.output import FortranOutputWriter
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "res_files.json")))
    w = FortranOutputWriter(str(tmp_path))
    for it in d["inputs"]:
        en = types.SimpleNamespace(**it["energies"])
        ob = types.SimpleNamespace(**{k: (np.array(v) if isinstance(v, list) else v)
                                      for k, v in it["observables"].items()})
        w.write_iteration_data(it["iteration"], en, ob, types.SimpleNamespace(x0dmp=it["x0dmp"]),
                               types.SimpleNamespace(epair=np.array(it["epair"])))
    for name, text in d["files"].items():
        with open(os.path.join(tmp_path, name), encoding="utf-8") as f:
            assert f.read() == text, name


def test_observables_layout_matches_header():
    """hfb.output's offsets into the hfb_observables output are the
    HFB_OBS_* values of include/hfb.h and tile the HFB_NOBS doubles."""
    from hfb import output
    txt = open(HEADER).read()
    enum = {k: int(v) for k, v in re.findall(r"HFB_OBS_(\w+)\s*=\s*(\d+)", txt)}
    nobs = int(re.search(r"HFB_NOBS\s*=\s*(\d+)", txt).group(1))
    names = {"pnr": "PNR", "cm": "CM", "pcm": "PCM", "rms": "RMS", "x2m": "X2M", "q20": "Q20", "q22": "Q22",
             "pnrtot": "PNRTOT", "cmtot": "CMTOT", "rmstot": "RMSTOT", "x2mtot": "X2MTOT", "q20tot": "Q20TOT",
             "q22tot": "Q22TOT", "q20T1": "Q20T1", "beta20tot": "BETA20", "beta22tot": "BETA22", "beta": "BETA",
             "gamma": "GAMMA", "dipole_isovector": "DIPOLE", "qmat": "QMAT"}
    assert nobs == output.HFB_NOBS
    used = np.zeros(nobs, dtype=int)
    for k, (off, shp) in output._OBS.items():
        assert enum[names[k]] == off, k
        used[off:off + int(np.prod(shp)) if shp else off + 1] += 1
    assert np.all(used == 1)


def test_sensitivity_parameters_and_rebuilt_forces():
    """The eleven Skyrme couplings of the force table and the two pairing
    strengths are the sensitivity parameters; W0 is the direction that moves
    t4 and b4p in proportion (its row is the chain rule of theirs); the
    forces the response solve rebuilds for one changed coupling equal the
    table's forces with that override."""
    from hfb import adjoint
    from hfb.forces import init_forces
    assert adjoint.SKYRME == ("t0", "t1", "t2", "t3", "x0", "x1", "x2", "x3", "t4", "b4p", "power")
    assert adjoint.PARAMS == adjoint.SKYRME + ("v0neut", "v0prot")
    base = init_forces(None, name="SLy4", ipair=5)
    th = adjoint.theta_of(base)
    assert set(adjoint.PARAMS) <= set(th) and th["W0"] == th["t4"]
    jac = adjoint._db_dtheta(base)
    for b in ("b4", "b4p"):
        w0 = jac["t4"].get(b, 0.0) + base.b4p / base.t4 * jac["b4p"].get(b, 0.0)
        assert jac["W0"].get(b, 0.0) == pytest.approx(w0, rel=1e-15)
    for name in ("t0", "x2", "t4", "b4p", "power", "W0"):
        v = th[name] * 1.01
        f1 = adjoint._forces_at(base, name, v)
        ov = adjoint.force_overrides(dict(force=dict(name="SLy4")), {name: v})["force"]["overrides"]
        f2 = init_forces(None, name="SLy4", ipair=5, overrides=ov)
        for b in ("b0", "b0p", "b1", "b1p", "b2", "b2p", "b3", "b3p", "b4", "b4p", "power"):
            assert getattr(f1, b) == pytest.approx(getattr(f2, b), rel=1e-14), (name, b)


def _prototypes():
    """name -> list of parameter declarations of every hfb_* prototype in
    include/hfb.h (comments removed, multi-line declarations joined)."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    txt = re.sub(r"//[^\n]*", " ", txt)
    out = {}
    for m in re.finditer(r"(?:int|const char\*|unsigned long long)\s+(hfb_\w+)\s*\(([^;{]*?)\)\s*;", txt, re.S):
        params = " ".join(m.group(2).split())
        out[m.group(1)] = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
    return out


def test_python_prototypes_match_the_header():
    """Every prototype the Python mirror declares has the header's number of
    parameters, and each parameter is of the same kind: a pointer for a
    pointer (device buffer, handle, stream, struct), double for double,
    long long for long long, int for int."""
    import ctypes as C
    from hfb import _lib
    protos = _prototypes()
    assert set(_lib._PROTOS) <= set(protos)
    for name, args in _lib._PROTOS.items():
        params = protos[name]
        assert len(params) == len(args), (name, params, args)
        for p, a in zip(params, args):
            if "*" in p or p.startswith(("hfb_ctx_t", "void* ")):
                kind = "ptr"
            elif p.startswith("double"):
                kind = "double"
            elif p.startswith("long long"):
                kind = "longlong"
            else:
                assert p.startswith("int"), (name, p)
                kind = "int"
            is_ptr = a is C.c_void_p or (isinstance(a, type) and issubclass(a, C._Pointer))
            py = ("ptr" if is_ptr else "double" if a is C.c_double else "longlong" if a is C.c_longlong
                  else "int" if a is C.c_int else repr(a))
            assert py == kind, (name, p, a)
