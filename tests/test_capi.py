"""The C ABI library loads on a CPU-only machine and exports every entry point
include/lbm_b200.h declares; without a GPU, creation fails cleanly."""
import ctypes
import re

import numpy as np
import pytest

from lbm_b200 import capi


def declared_functions():
    text = open(capi.HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(capi.SIGNATURES)


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_create_rejects_bad_descriptor():
    d = capi.LbmDesc()
    d.lattice = 20
    h = ctypes.c_void_p()
    rc = capi.lib().lbm_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == capi.LBM_ERR_ARGUMENT
    assert b"lattice" in capi.lib().lbm_last_error(None)


def test_reference_mode_requires_d3q19():
    d = capi.LbmDesc()
    d.lattice, d.bc_mode, d.tau = 27, capi.BC_REFERENCE, 0.8
    h = ctypes.c_void_p()
    rc = capi.lib().lbm_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == capi.LBM_ERR_ARGUMENT
    assert b"D3Q19" in capi.lib().lbm_last_error(None)


def test_null_handle_calls_fail_cleanly():
    L = capi.lib()
    assert L.lbm_step(None, 1) == capi.LBM_ERR_ARGUMENT
    assert L.lbm_destroy(None) == capi.LBM_ERR_ARGUMENT
    assert L.lbm_halo_define(None, 0, 0, None, None) == capi.LBM_ERR_ARGUMENT
    assert L.lbm_halo_pack(None, 0, None) == capi.LBM_ERR_ARGUMENT
    assert L.lbm_halo_unpack(None, 0, None) == capi.LBM_ERR_ARGUMENT
    assert L.lbm_get_phase(None, None) == capi.LBM_ERR_ARGUMENT
    assert L.lbm_last_error(None)


def test_create_without_gpu_reports_no_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lbm_b200 import Engine
    topo = {"coords": np.array([[0, 0, 0], [0, 0, 1]]), "kind": np.zeros(2, np.uint8),
            "inlet": np.zeros(0), "inlet_normal": np.zeros(3), "wall": np.zeros(0),
            "nearwall": np.zeros(0), "nearwall_normal": np.zeros((0, 3))}
    with pytest.raises(capi.LbmError) as ei:
        Engine(topo, tau=0.8)
    assert ei.value.code == capi.LBM_ERR_NO_DEVICE


STRUCTS = {"LbmDesc": "lbm_desc", "LbmAdjointDesc": "lbm_adjoint_desc", "LbmAdjointResult": "lbm_adjoint_result",
           "LbmOpening": "lbm_opening", "LbmVoxelDesc": "lbm_voxel_desc", "LbmPulseDesc": "lbm_pulse_desc",
           "LbmEquation": "lbm_equation", "LbmConfig": "lbm_config"}


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes structure of the binding has the size and field offsets a C
    compiler gives the header's typedef (a program built against
    include/lbm_b200.h prints them)."""
    import os
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "lbm_b200.h"', "int main(void) {"]
    want = []
    for py, c in STRUCTS.items():
        cls = getattr(capi, py)
        lines.append('printf("%%zu\\n", sizeof(%s));' % c)
        want.append(ctypes.sizeof(cls))
        for name, _ in cls._fields_:
            lines.append('printf("%%zu\\n", offsetof(%s, %s));' % (c, name))
            want.append(getattr(cls, name).offset)
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.dirname(capi.HEADER_PATH), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == want


def header_prototypes():
    """{name: (return type, [parameter declarations])} from the header."""
    text = open(capi.HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"^\s*#.*$", "", text, flags=re.M)  # preprocessor lines
    protos = {}
    for ret, name, params in re.findall(r"([A-Za-z_][\w\s\*]*?)\b(lbm_[a-z_]+)\s*\(([^;{]*?)\)\s*;", text):
        p = [x.strip() for x in params.split(",")] if params.strip() not in ("", "void") else []
        protos[name] = (" ".join(ret.split()), p)
    return protos


def c_kind(decl):
    """The kind of value a C declaration passes: pointer or an integer or
    floating type of a given size."""
    if "*" in decl or "[" in decl:  # an array parameter is a pointer
        return "pointer"
    t = decl.replace("const ", "").split()[0]
    return {"int": "i32", "int32_t": "i32", "uint32_t": "u32", "int64_t": "i64", "size_t": "u64",
            "double": "f64", "float": "f32"}[t]


def ctypes_kind(t):
    if t in (ctypes.c_void_p, ctypes.c_char_p) or (isinstance(t, type) and issubclass(t, ctypes._Pointer)):
        return "pointer"
    return {ctypes.c_int32: "i32", ctypes.c_uint32: "u32", ctypes.c_int64: "i64", ctypes.c_uint64: "u64",
            ctypes.c_double: "f64", ctypes.c_float: "f32"}[t]


def test_binding_signatures_match_header_prototypes():
    """Each entry point's ctypes signature passes the same number and kinds of
    arguments as its prototype in include/lbm_b200.h, and its return value
    has the prototype's kind: a parameter added on one side only fails
    here, without a GPU."""
    protos = header_prototypes()
    assert sorted(protos) == sorted(capi.SIGNATURES)
    for name, (res, args) in capi.SIGNATURES.items():
        ret, params = protos[name]
        assert len(params) == len(args), (name, params)
        for decl, t in zip(params, args):
            assert c_kind(decl) == ctypes_kind(t), (name, decl, t)
        if ret == "void":
            assert res is None, (name, res)
        else:
            assert ("pointer" if "*" in ret else c_kind(ret)) == ctypes_kind(res), (name, ret, res)
