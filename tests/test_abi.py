"""The C ABI without a GPU: the library loads, exports every declared entry point, its structures match the
header field for field, and the host-only analysis works."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from gridsim_b200 import _abi, synthetic
from tests.conftest import ROOT, golden_model

HEADER = os.path.join(ROOT, "include", "gridsim_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gs_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = _abi.load_library()
    names = declared_functions()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), f"{name} is declared in the header but not exported"
    assert set(names) == set(_abi.EXPORTS), "the ctypes table and the header disagree"


def test_struct_layouts_match_the_header(tmp_path):
    structs = {"gs_grid_desc": _abi.GridDesc, "gs_pf_opts": _abi.PfOpts, "gs_pf_result": _abi.PfResult,
               "gs_n1_result": _abi.N1Result, "gs_grid_info": _abi.GridInfo, "gs_ctx_opts": _abi.CtxOpts,
               "gs_serve_opts": _abi.ServeOpts, "gs_request": _abi.Request, "gs_response": _abi.Response,
               "gs_serve_stats": _abi.ServeStats, "gs_multi_stats": _abi.MultiStats, "gs_schedule": _abi.Schedule}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-o", str(exe), str(src)])
    got = dict(line.split() for line in subprocess.check_output([str(exe)]).decode().splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, f"{cname}.{fname}"


def test_status_strings_and_defaults():
    lib = _abi.load_library()
    assert lib.gs_abi_version() == 2
    assert lib.gs_status_str(_abi.GS_ERR_OOM) == b"out of device memory"
    o = _abi.PfOpts()
    lib.gs_pf_opts_default(ctypes.byref(o))
    d = _abi.default_opts()
    for f, _ in _abi.PfOpts._fields_:
        if f != "reserved":
            assert getattr(o, f) == getattr(d, f), f


def test_context_on_a_machine_without_a_device_reports_no_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = _abi.load_library()
    h = ctypes.c_void_p()
    o = _abi.CtxOpts()
    o.probe_timeout_ms = 20000
    rc = lib.gs_ctx_create(0, ctypes.byref(o), ctypes.byref(h))
    assert rc in (_abi.GS_ERR_NO_DEVICE, _abi.GS_ERR_TIMEOUT)
    assert not h.value


@pytest.mark.parametrize("name", ["case9", "case118", "case300"])
def test_host_analysis_sizes(name):
    import oracle
    m, _ = golden_model(name)
    info = _abi.GridInfo()
    d = m.desc()
    assert _abi.load_library().gs_analyze_host(ctypes.byref(d), ctypes.byref(info)) == _abi.GS_OK
    n_pq = int(np.sum(m.bus_type == 1))
    assert info.m == (m.n_bus - 1) + n_pq
    rp, ci, _, _ = oracle.jacobian(m)
    assert info.nnz_j == len(ci)          # the superset pattern is the reference's pattern here
    assert info.nnz_lu >= info.nnz_j      # static pivots: L + U covers J plus fill
    assert info.n_levels >= 1 and info.lu_flops >= 0


def test_host_analysis_refuses_bad_descriptors():
    m = synthetic.config_grid(0, 0)
    m.br_to[0] = m.br_from[0]  # a branch from a bus to itself
    info = _abi.GridInfo()
    d = m.desc()
    assert _abi.load_library().gs_analyze_host(ctypes.byref(d), ctypes.byref(info)) == _abi.GS_ERR_INVALID_ARG
