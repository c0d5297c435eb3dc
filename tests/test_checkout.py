"""The Python 3 port of the reference's flow-case generator
(shared_cfd_b200/checkout.py): its assembly mechanics on a miniature store,
the GPU architecture value, and, when SCFD_REFERENCE names a reference
checkout, the real store on the forward-step samples."""
import os
import shutil

import numpy as np
import pytest

from shared_cfd_b200 import cases, checkout
from shared_cfd_b200 import formats as F

from conftest import REFERENCE


def _write(root, rel, text):
    p = os.path.join(root, rel)
    os.makedirs(os.path.dirname(p), exist_ok=True)
    with open(p, "w") as fh:
        fh.write(text)


def _mini_store(root):
    """A store/ with the fragment layout of the reference and marker contents."""
    w = lambda rel, text: _write(root, "store/" + rel, text)
    w("core/Makefile.main", "all: main\n#core rules\n")
    w("core/Makefile.var", "")
    w("core/Makefile.foot", "#foot\n")
    w("core/main.part_top.f90", "program main\n")
    w("core/main.part_init.f90", "   call set_MPI\n")
    w("core/main.part_main.f90", "   call core_main\n")
    w("core/main.head.f90", "   implicit none\n")
    w("core/main.body.raw.f90", "   i=step_res+1\npart_primitive\n   do while(check_convergence(i,step_res))\n")
    w("core/main.foot.f90", "      i=i+1\n   end do\nend program main\n")
    w("core/n_grid.raw.f90", "Nplane = NPLANE\nni=(/NumI/)\nnj=(/NumJ/)\nNIMAX NJMAX NumY NV GridFileName\n")
    w("core/control.part.inp", "#core controls\n")
    w("architecture/PC/Makefile.head", "arc=mod_mpi_dummy.o\n")
    w("architecture/PC/mod_mpi_dummy.f90", "module mod_mpi\nend module mod_mpi\n")
    w("dim/2d/geometry.f90", "module geometry\nend module geometry\n")
    w("time_step/global/set_dt.f90", "subroutine set_dt\nend subroutine set_dt\n")
    w("time_scheme/euler/time_euler_viscous.raw.f90", "q = qp + DT_LOCAL_GLOBAL\n")
    w("time_scheme/euler/main.main.raw.f90", "part_main\n      call calc_next_step\n")
    w("high_order/muscl/muscl.f90", "module half_value\nend module half_value\n")
    w("therm_lib/ideal/thermal_model.raw.f90", "kappa=KAPPA rgas=RGAS nu=NU\n")
    w("therm_lib/ideal/main.part_primitive.f90", "   call set_w\n")
    w("viscosity/non-viscous/viscous.f90", "subroutine set_TGv\nend subroutine set_TGv\n")
    w("cond/core/condition.head.f90", "subroutine set_BC(step)\n")
    w("cond/core/condition.tail.f90", "end subroutine set_BC\n")
    w("cond/core/gen_cond.py", "# Python 2 original, replaced by the port\n")
    w("cond/no-nV/condition.tail.f90", "end subroutine set_BC\n")


def _case_root(tmp_path, arch, orientation=0):
    root = str(tmp_path)
    _mini_store(root)
    planes = cases.forward_step(orientation, n=6).planes
    with open(os.path.join(root, "fs.x"), "w") as fh:
        fh.write(F.format_plot3d(planes))
    _write(root, "checkout.inp",
           "grid file name    : fs.x #Grid file name (*.x)\n"
           "NumOfProcessors   : %s  #architecture\n"
           "dimension         : 0  #two dimension(0)/axi-symmetry(1)\n"
           "time step         : 0  #global(0)/local(1)\n"
           "time scheme       : 0  #Euler(0)\n"
           "high order scheme : 1  #Up Wind(0)/MUSCL(1)\n"
           "viscosity         : 0  #non-viscous flow(0)/viscous flow(1)\n"
           "thermal model     : 0  #Ideal Gas(0)\n" % arch)
    return root, planes


def test_mini_store_personal_computer(tmp_path):
    root, planes = _case_root(tmp_path, "0")
    sel = checkout.checkout_flow(root, log=lambda *a: None)
    out = os.path.join(root, "checkout")
    read = lambda n: open(os.path.join(out, n)).read()
    assert sel["architecture"] == "PC" and sel["nplane"] == 2
    assert read("main.f90") == ("program main\n   implicit none\n   call set_MPI\n   i=step_res+1\n   call set_w\n"
                                "   do while(check_convergence(i,step_res))\n   call core_main\n"
                                "      call calc_next_step\n      i=i+1\n   end do\nend program main\n")
    assert read("time_euler_viscous.f90") == "q = qp + dt_grbl\n"
    assert read("thermal_model.f90") == "kappa=1.4d0 rgas=287d0 nu=1.6d-5\n"
    ni = [xh.shape[0] - 1 for xh, _ in planes]
    nj = [xh.shape[1] - 1 for xh, _ in planes]
    assert read("n_grid.f90").splitlines()[:3] == ["Nplane = 2", "ni=(/%d,%d/)" % tuple(ni), "nj=(/%d,%d/)" % tuple(nj)]
    assert read("Makefile") == "arc=mod_mpi_dummy.o\nall: main\n#core rules\n#foot\n"
    recs, tsm = F.connectivity(F.read_plot3d(os.path.join(root, "fs.x")))
    assert F.read_cut_copro(os.path.join(out, "cut_copro000.inp")) == [list(r) for r in recs]
    cond = read("condition.raw.f90")
    assert cond.startswith("subroutine set_BC(step)\n   integer,parameter::MaxMPIcomm = 0\n")
    for p, sides in enumerate(tsm):
        for lo, hi in sides[0][0] + sides[0][1]:
            assert "do j=max(%5i,nys(plane)),min(nye(plane),%5i)" % (lo, hi) in cond
    # templates, parts and the Python generator files are gone
    for n in os.listdir(out):
        if n in ("condition.raw.f90", "control.raw.inp"):
            continue  # the user's condition.f90 / control.inp are made from these
        assert ".raw." not in n and not n.startswith("main.part_") and not n.endswith(".py"), n
    assert sorted(os.listdir(os.path.join(out, "grid"))) == ["fs.x"]


def test_mini_store_gpu_architecture(tmp_path):
    root, _ = _case_root(tmp_path, "GPU")
    sel = checkout.checkout_flow(root, log=lambda *a: None)
    out = os.path.join(root, "checkout")
    read = lambda n: open(os.path.join(out, n)).read()
    assert sel["architecture"] == "GPU"
    main = read("main.f90")
    # the GPU time-loop body replaces the scheme's own
    assert "call scfd_gpu_step(i)" in main and "call calc_next_step" not in main
    mk = read("Makefile")
    assert "-lscfd_b200" in mk and "scfd_gpu_driver.o" in mk and mk.index("all: main") < mk.index("scfd_b200_iface.o:")
    drv = read("scfd_gpu_driver.f90")
    assert "GPU_" not in drv
    assert "desc%scheme = 0" in drv and "desc%recon = 1" in drv and "desc%kappa = 1.4d0" in drv
    assert "use half_value, only: phi_mus, k_mus" in drv and "desc%k_mus = k_mus" in drv
    assert read("scfd_gpu_chem.f90").startswith("! no chemistry tables")
    assert not os.path.exists(os.path.join(out, "scfd_gpu_chem.chemkin.f90"))
    bc = read("scfd_gpu_bc.raw.f90")
    _, tsm = F.connectivity(F.read_plot3d(os.path.join(root, "fs.x")))
    n = sum(len(r) for sides in tsm for c in sides for r in c)
    assert bc.count("SCFD_BC_EXTRAP, 0, 0d0)") == n and "ierr = scfd_set_bc(ctx, b, %d)" % n in bc
    assert "module scfd_b200_iface" in read("scfd_b200_iface.f90")


def test_unported_and_unsupported_choices_are_refused(tmp_path):
    root, _ = _case_root(tmp_path, "4")
    with pytest.raises(checkout.CheckoutError):
        checkout.checkout_flow(root, log=lambda *a: None)
    txt = open(os.path.join(root, "checkout.inp")).read().replace(": 4 ", ": GPU ").replace(
        "time scheme       : 0", "time scheme       : 1")
    with open(os.path.join(root, "checkout.inp"), "w") as fh:
        fh.write(txt)
    os.makedirs(os.path.join(root, "store/time_scheme/RK2"), exist_ok=True)
    _write(root, "store/time_scheme/RK2/time_RK2_viscous.raw.f90", "DT_LOCAL_GLOBAL\n")
    with pytest.raises(checkout.CheckoutError):
        checkout.checkout_flow(root, log=lambda *a: None)


def test_ckinterp_counts():
    assert checkout.ckinterp(cases.seeded_chem_inp()) == (3, 9, 19)
    txt = ("elements\nH O\nend\nspecies\nH2 O2\n! comment\nH2O\nend\nthermo\nx\nend\n"
           "reactions\nH2+O2=H2O2 1 0 0\n DUPLICATE\nH+O=OH 1 0 0\n LOW /1 2 3/\nend\n")
    assert checkout.ckinterp(txt) == (2, 3, 2)


@pytest.mark.skipif(not REFERENCE or not os.path.isdir(REFERENCE),
                    reason="SCFD_REFERENCE does not name a reference checkout")
@pytest.mark.parametrize("sample", ["no06.step_flow", "no07.step_flow2", "no08.step_flow3", "no09.step_flow4"])
@pytest.mark.parametrize("arch", ["0", "GPU"])
def test_reference_store_forward_step_samples(tmp_path, sample, arch):
    """The real store on the forward-step samples: every user-boundary loop
    header of the generated condition.raw.f90 is the one the sample's
    condition.f90 (the reference generator's output, filled in by hand) holds,
    in the same order; the GPU value gives a program whose time loop calls the
    library."""
    root = str(tmp_path)
    shutil.copytree(os.path.join(REFERENCE, "store"), os.path.join(root, "store"))
    src = os.path.join(REFERENCE, "sample", sample)
    for n in os.listdir(src):
        if n.endswith(".x") or n == "checkout.inp":
            shutil.copyfile(os.path.join(src, n), os.path.join(root, n))
    txt = open(os.path.join(root, "checkout.inp")).read().splitlines(keepends=True)
    txt[1] = "NumOfProcessors   : %s  #architecture\n" % arch
    with open(os.path.join(root, "checkout.inp"), "w") as fh:
        fh.write("".join(txt))
    checkout.checkout_flow(root, log=lambda *a: None)
    out = os.path.join(root, "checkout")
    gen = [ln.strip() for ln in open(os.path.join(out, "condition.raw.f90")) if ln.strip().startswith("do ")]
    ref = [ln.strip() for ln in open(os.path.join(src, "condition.f90"))
           if ln.strip().startswith("do ") and "max(" in ln and "nys(plane)" in ln or "nxs(plane)),min(nxe" in ln]
    ref = [r.strip() for r in ref]
    assert [g for g in gen if g in ref] == ref[:len([g for g in gen if g in ref])]
    assert set(ref) <= set(gen)
    main = open(os.path.join(out, "main.f90")).read()
    assert ("call scfd_gpu_step(i)" in main) == (arch == "GPU")
    assert os.path.exists(os.path.join(out, "cut_copro000.inp"))
