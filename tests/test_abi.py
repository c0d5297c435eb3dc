"""The C ABI: every function include/scfd_b200.h declares is exported by the
CUDA library (and, with the orc_ prefix, by the CPU restatement); struct
layouts agree between C and the ctypes mirror; argument checking needs no GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from shared_cfd_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "scfd_b200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|void\*)\s+scfd_(\w+)\s*\(", txt, flags=re.M)))


def cuda_lib_path():
    from shared_cfd_b200 import build
    build.build()
    return build.OUT


def test_header_declares_the_bound_functions():
    names = declared()
    assert set(abi.SIGNATURES) <= set(names), set(abi.SIGNATURES) - set(names)


def test_cuda_library_exports_every_declared_symbol():
    lib = C.CDLL(cuda_lib_path())
    for n in declared():
        assert hasattr(lib, "scfd_" + n), n


def test_oracle_exports_same_entry_points(orc_raw):
    # scfd_rms_noalloc works on device arrays only; the CPU restatement has no
    # counterpart of it
    for n in declared():
        if n.endswith("noalloc"):
            continue
        assert hasattr(orc_raw, "orc_" + n), n


def test_struct_sizes_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include "%s"\nint main(void){printf("%%zu %%zu %%zu %%zu %%zu\\n",'
                   'sizeof(scfd_desc),sizeof(scfd_bc),sizeof(scfd_chem),sizeof(scfd_stats),'
                   'sizeof(scfd_reactor_desc));printf("%%zu %%zu\\n",sizeof(scfd_cea_data),'
                   'sizeof(scfd_cea_info));return 0;}\n' % HEADER)
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-o", str(exe), str(src)])
    out = [int(v) for v in subprocess.check_output([str(exe)]).split()]
    assert out == [C.sizeof(abi.Desc), C.sizeof(abi.BC), C.sizeof(abi.Chem), C.sizeof(abi.Stats),
                   C.sizeof(abi.ReactorDesc), C.sizeof(abi.CeaData), C.sizeof(abi.CeaInfo)]


def test_create_rejects_bad_descriptors_without_gpu():
    lib = abi.Bound(C.CDLL(cuda_lib_path()), "scfd_")
    assert lib.abi_version() == abi.ABI_VERSION
    d = abi.Desc()
    ctx = C.c_void_p()
    d.abi_version = 99
    assert lib.create(C.byref(d), C.byref(ctx)) == abi.E_ARG
    d.abi_version = abi.ABI_VERSION
    d.nplane, d.ny, d.ni[0], d.nj[0] = 1, 1, 8, 8
    d.scheme = 7
    assert lib.create(C.byref(d), C.byref(ctx)) == abi.E_UNSUPPORTED
    d.scheme = abi.SCHEME_LUSGS
    d.thermo = abi.THERMO_CHEMKIN_REACTIVE
    d.dt_mode = abi.DT_LOCAL
    d.ny = 9
    assert lib.create(C.byref(d), C.byref(ctx)) == abi.E_UNSUPPORTED   # checkout_flow.py:231-233
    d.thermo, d.dt_mode, d.ny = abi.THERMO_IDEAL, abi.DT_GLOBAL, 1
    assert lib.create(C.byref(d), C.byref(ctx)) == 0
    b = abi.BC()
    b.plane, b.side, b.first, b.last, b.kind = 1, abi.SIDE_ILO, 1, 9, abi.BC_EXTRAP
    assert lib.set_bc(ctx, C.byref(b), 1) == abi.E_ARG                 # range beyond nj
    b.last = 8
    assert lib.set_bc(ctx, C.byref(b), 1) == 0
    assert lib.commit(ctx) == abi.E_STATE                              # geometry missing
    assert lib.step(ctx, 1, None) == abi.E_STATE
    assert lib.destroy(ctx) == 0


def test_library_fails_loudly_when_missing(tmp_path):
    from shared_cfd_b200 import solver
    with pytest.raises(solver.CudaLibraryMissing):
        solver.load_library(str(tmp_path / "nope.so"))
