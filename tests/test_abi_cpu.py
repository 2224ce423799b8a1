"""CPU-only checks of the product boundary: the C-ABI library loads and exports
every entry point include/twos.h declares, the ctypes structures match the C
layouts, and the executables keep the reference's usage/runtime exit codes
(wih_twos.cpp:103-135, 1860-1863; study.cpp/adjoint.cpp serve framing)
without touching a GPU.
"""
import ctypes

import numpy as np
import re
import subprocess

import pytest

from conftest import GOLDEN, PKG, REPO


def _declared():
    text = (REPO / "include" / "twos.h").read_text()
    return sorted(set(re.findall(r"\b(twos_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lib_built):
    from twos_b200 import _abi
    lib = ctypes.CDLL(str(_abi.LIB_PATH))
    declared = _declared()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_abi.EXPORTED)


def test_abi_version_and_layouts(lib_built, tmp_path):
    """Every ctypes field offset and struct size equals the C header's."""
    from twos_b200 import _abi
    L = _abi.load()
    assert L.twos_abi_version() == _abi.ABI_VERSION == 2
    structs = {"twos_source_term": _abi.SourceTerm, "twos_request": _abi.Request,
               "twos_site_result": _abi.SiteResult, "twos_summary": _abi.Summary, "twos_mesh_info": _abi.MeshInfo,
               "twos_tuning": _abi.Tuning, "twos_design_params": _abi.DesignParams,
               "twos_design_step": _abi.DesignStep, "twos_rqmc_params": _abi.RqmcParams,
               "twos_validate_params": _abi.ValidateParams}
    # Result rows read as numpy structured arrays: field offsets and sizes.
    dtypes = {"twos_site_result": _abi.SITE_DTYPE, "twos_gradient_result": _abi.GRADIENT_DTYPE,
              "twos_diff_result": _abi.DIFF_DTYPE, "twos_diff_stats": _abi.DIFF_STATS_DTYPE,
              "twos_cert_sample": _abi.CERT_SAMPLE_DTYPE, "twos_validate_stage": _abi.VALIDATE_STAGE_DTYPE,
              "twos_design_step": _abi.DESIGN_DTYPE}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "twos.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    for cname, dt in dtypes.items():
        lines.append(f'printf("np.{cname} %zu\\n", sizeof({cname}));')
        for f in dt:
            lines.append(f'printf("np.{cname}.{f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)
    for cname, dt in dtypes.items():
        d = np.dtype(dt, align=True)
        # The package builds these dtypes unaligned, so they must need no padding.
        assert np.dtype(dt).itemsize == d.itemsize, cname
        assert int(got[f"np.{cname}"]) == d.itemsize, cname
        for f in dt:
            assert int(got[f"np.{cname}.{f[0]}"]) == d.fields[f[0]][1], (cname, f[0])


def test_request_validation_without_gpu(lib_built):
    from twos_b200 import _abi
    from twos_b200.mesh import Config
    L = _abi.load()
    cfg = Config(walks=1)
    req = cfg.to_request()
    # A null mesh is a usage error before any device work.
    rc = L.twos_estimate(None, ctypes.byref(req), None, 0, None, 0, None, None)
    assert rc == _abi.ERR_USAGE


def _exe(name):
    return str(PKG / "_build" / name)


def test_cli_usage_errors_exit_2(lib_built, tmp_path):
    r = subprocess.run([_exe("wih_twos")], capture_output=True, text=True)
    assert r.returncode == 2 and "--mesh, --points, --output, and --summary are required" in r.stderr
    base = ["--mesh", "m.ply", "--points", "p.csv", "--output", "o.csv", "--summary", "s.json"]
    for extra, msg in [(["--walks", "1"], "invalid numeric option"),
                       (["--bogus", "1"], "unknown option --bogus"),
                       (["--mode", "diffwos"], "Differential WoS requires --cavities"),
                       (["--grid", "3,x,4"], "--grid must have the form NX,NY,NZ"),
                       (["--cavities", "c.csv"], "invalid numeric option"),
                       (["--walks"], "missing value for --walks")]:
        r = subprocess.run([_exe("wih_twos")] + base + extra, capture_output=True, text=True)
        assert r.returncode == 2, (extra, r.stderr)
        assert msg in r.stderr


def test_cli_bad_mesh_is_runtime_error(lib_built, tmp_path):
    bad = tmp_path / "bad.ply"
    bad.write_text("ply\nformat binary_little_endian 1.0\nelement vertex 3\nend_header\n")
    pts = tmp_path / "p.csv"
    pts.write_text("0,0,0\n")
    r = subprocess.run([_exe("wih_twos"), "--mesh", str(bad), "--points", str(pts), "--output",
                        str(tmp_path / "o.csv"), "--summary", str(tmp_path / "s.json")], capture_output=True,
                       text=True)
    assert r.returncode == 1
    assert "fatal: expected a nonempty ASCII triangle PLY mesh" in r.stderr
    tri = tmp_path / "quad.ply"
    tri.write_text("ply\nformat ascii 1.0\nelement vertex 4\nproperty double x\nproperty double y\n"
                   "property double z\nelement face 1\nproperty list uchar int vertex_indices\nend_header\n"
                   "0 0 0\n1 0 0\n0 1 0\n1 1 0\n4 0 1 2 3\n")
    r = subprocess.run([_exe("wih_twos"), "--mesh", str(tri), "--points", str(pts), "--output",
                        str(tmp_path / "o.csv"), "--summary", str(tmp_path / "s.json")], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "expected valid triangular PLY faces" in r.stderr


def test_cli_grid_modes_are_refused(lib_built, tmp_path):
    pts = tmp_path / "p.csv"
    pts.write_text("0,0,0\n")
    r = subprocess.run([_exe("wih_twos"), "--mesh", str(GOLDEN / "missing.ply"), "--points", str(pts),
                        "--output", str(tmp_path / "o.csv"), "--summary", str(tmp_path / "s.json"), "--mode",
                        "voxel"], capture_output=True, text=True)
    assert r.returncode == 1 and "not provided by the TWoS B200 backend" in r.stderr


def test_serve_framing_errors_exit_2(lib_built):
    for payload in ["abc\n", "0\n", "201\n", "3\nonly-one-line\n"]:
        r = subprocess.run([_exe("wih_adjoint"), "--serve"], input=payload, capture_output=True, text=True)
        assert r.returncode == 2, payload
    r = subprocess.run([_exe("wih_adjoint"), "--serve"], input="", capture_output=True, text=True)
    assert r.returncode == 0


def test_serve_usage_error_answers_done_2(lib_built):
    payload = "3\nwih_adjoint\n--walks\n1\n"
    r = subprocess.run([_exe("wih_adjoint"), "--serve"], input=payload, capture_output=True, text=True)
    assert r.stdout.strip() == "DONE 2" and r.returncode == 2


def test_product_does_not_import_oracle():
    # The product package and library sources never reference the oracle.
    pattern = re.compile(r"import\s+oracle|from\s+oracle|libtwos_oracle|oracle/|oracle\.")
    for p in list((PKG / "twos_b200").glob("*.py")) + list((PKG / "csrc").glob("*")) + [PKG / "build.py"]:
        assert not pattern.search(p.read_text()), p
