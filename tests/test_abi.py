"""The C-ABI library loads without a GPU and exports every function the
public headers declare; the layout contract matches gpu_layout.rs. No compute
calls are made here."""
import os
import re
import subprocess

import numpy as np

from lucida_b200 import layout as L
from lucida_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("luc_cuda.h", "lucida_layout.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(luc_[a-z0-9_]+)\s*\(", text))
    return names


def test_every_declared_symbol_is_exported_and_bound():
    decl = declared_functions()
    assert "luc_render" in decl and "luc_upload_scene" in decl and "luc_lbvh_build" in decl
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (luc_[a-z0-9_]+)", out))
    assert decl <= exported, sorted(decl - exported)
    assert decl == set(native.exported_symbols()), sorted(decl ^ set(native.exported_symbols()))
    lib = native.lib()
    for name in decl:
        assert getattr(lib, name) is not None


def test_layout_contract():
    lib = native.lib()
    assert lib.luc_layout_version() == 1
    sizes = [lib.luc_sizeof(i) for i in range(9)]
    assert sizes == [80, 64, 64, 32, 16, 32, 64, 160, 64]
    assert [L.MATERIAL.itemsize, L.PRIMITIVE.itemsize, L.LIGHT.itemsize, L.VERTEX_ATTR.itemsize,
            L.TRIANGLE.itemsize, L.BVH_NODE.itemsize, L.ACCUM.itemsize] == sizes[:7]
    # gpu_layout.rs:993-1166 offsets
    assert L.MATERIAL.fields["emissive"][1] == 16 and L.MATERIAL.fields["eta"][1] == 48
    assert L.PRIMITIVE.fields["kind"][1] == 28 and L.PRIMITIVE.fields["normal"][1] == 48
    assert L.ACCUM.fields["radiance_sq"][1] == 48 and L.Uniforms.tlas_root.offset == 144


def test_errors_without_a_device_are_reported_not_raised_in_c():
    import ctypes as C
    lib = native.lib()
    h = C.c_void_p()
    rc = lib.luc_create(0, C.byref(h))
    try:
        import torch
        has = torch.cuda.is_available()
    except Exception:
        has = False
    if not has:
        assert rc == -1 and not h.value  # GpuError::NoAdapter
    elif rc == 0:
        lib.luc_destroy(h)
    assert lib.luc_render(None, None, 1, 1, 0, None, None) == -4  # null context -> Validation
