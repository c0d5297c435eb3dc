"""Python 3 port of the reference's flow-case generator, with a GPU
architecture.

    cd <reference checkout>      # the directory holding store/, checkout.inp, the grid
    python -m shared_cfd_b200.checkout

The reference assembles a Fortran program from fragments (checkout.py ->
store/checkout/checkout_flow.py with checkout_utility.py, and the boundary
generator store/cond/core/{gen_cond,read_plot3d,set_cond_var,mod_cond,
out_cond}.py), under Python 2.  This module does the same work under Python 3
and writes the same checkout/ directory: every line of checkout.inp selects
fragment directories under store/, whose files are copied in ("engaged"), whose
main.part_* / control.part.inp / Makefile.* parts are concatenated, and whose
*.raw.* templates get their placeholders replaced.

One value is added to the architecture line ("NumOfProcessors"), next to 0
(personal computer), > 0 (M-system, MPI) and < 0 (V-system): `GPU` selects the
B200 variant.  It engages the personal-computer fragments (single process, all
planes local) and then the fragments of shared_cfd_b200/store/architecture/GPU:
a Makefile.head that links libscfd_b200.so, the iso_c_binding module of
include/scfd_b200.h, a driver module that builds the device context from the
Fortran module arrays on the first step and runs each physical step through
scfd_step, and the time-loop body main.main.gpu.f90 that replaces the time
scheme's own main.main*.f90.  The time scheme, dimension, thermal model and
the rest still select their fragments (module arrays, set-up, I/O, boundary
templates) as in the reference; the arithmetic of the time loop runs on the
GPU.

Not ported: the M-system (> 0) path, which splits planes over MPI ranks with
store/architecture/SC/generate_proc_grid.py; a positive value is refused with
a message.
"""
import argparse
import os
import shutil
import sys

from . import formats as F

HERE = os.path.dirname(os.path.abspath(__file__))
GPU_STORE = os.path.join(HERE, "store")

# the part files whose contents are concatenated over all engaged fragments
# (checkout_flow.py:25-35)
PARTS = ["control.part.inp", "Makefile.main", "Makefile.var", "main.part_top.f90", "main.part_variable.f90",
         "main.part_init.f90", "main.part_point_implicit.f90", "main.part_primitive.f90", "main.part_main.f90"]


class CheckoutError(RuntimeError):
    pass


class Generator:
    """State of one run: the checkout directory and the concatenated parts."""

    def __init__(self, root, out="checkout", log=print):
        self.root = os.path.abspath(root)
        self.out = os.path.join(self.root, out)
        self.parts = {p: "" for p in PARTS}
        self.log = log

    # ---- checkout_utility.py ------------------------------------------------
    def path(self, name):
        return os.path.join(self.out, name)

    def engage(self, place, store=None):
        """Copy the files of store/<place> into the checkout and move the part
        files' contents into the concatenated parts (checkout_utility.py:46-50)."""
        src = os.path.join(store or os.path.join(self.root, "store"), place)
        if not os.path.isdir(src):
            raise CheckoutError("no fragment directory %s" % src)
        for name in sorted(os.listdir(src)):
            f = os.path.join(src, name)
            if os.path.isfile(f):
                shutil.copyfile(f, self.path(name))
        for name in PARTS:
            if os.path.exists(self.path(name)):
                self.parts[name] += self.take(name)

    def take(self, name):
        """file_to_str: the file's text; the file is removed."""
        with open(self.path(name)) as fh:
            text = fh.read()
        os.remove(self.path(name))
        return text

    def raw2pro(self, raw, pro, fromto):
        """Placeholder replacement line by line, in order; the template is
        removed (checkout_utility.py:18-27)."""
        with open(self.path(raw)) as fr, open(self.path(pro), "w") as fw:
            for line in fr:
                for a, b in fromto:
                    line = line.replace(a, b)
                fw.write(line)
        os.remove(self.path(raw))

    def append(self, fh, name):
        """append_file_to_file: the file's text onto fh; the file is removed."""
        fh.write(self.take(name))


def read_control_next(fh):
    """The value after ':' of the next line, up to a '#' comment
    (checkout_utility.py:29-35)."""
    s = fh.readline()
    if "#" in s:
        return s[s.index(":") + 1:s.index("#") - 1].strip()
    return s[s.index(":") + 1:].strip()


def read_control_next_int(fh, what):
    v = read_control_next(fh)
    try:
        return int(v)
    except ValueError:
        raise CheckoutError("odd input at %s: %r" % (what, v)) from None


# ---- store/cond/core/out_cond.py -------------------------------------------
def out_cond(g, tsm, max_mpi_comm, aboutnv):
    """condition.raw.f90: condition.head.f90, the user-boundary loops of every
    plane side that no block interface covers, condition.tail.f90."""
    nv = aboutnv == "with-nV"
    out = [g.take("condition.head.f90")]
    out.append("   integer,parameter::MaxMPIcomm = %i\n\n" % max_mpi_comm)
    out.append("   call section_exchange\n")
    out.append("   call MPI_COMMUNICATIONS_CUT_LINE\n\n")
    for direction in ("i", "j"):
        if direction == "i":
            out.append("\n   !boundary right and left\n   do plane=nps,npe\n      select case(plane)")
        else:
            out.append("\n   !boundary upper and lower\n   do plane=nps,npe\n      select case(plane)")
        for p, sides in enumerate(tsm):
            lo, hi = sides[0 if direction == "i" else 1]
            out.append("\n      case(%3i)" % (p + 1))
            if direction == "i":
                if lo:
                    out.append("\n         if(gx(plane) .eq. 1) then\n            !i=1/2")
                    for a, b in lo:
                        out.append("\n            do j=max(%5i,nys(plane)),min(nye(plane),%5i)"
                                   "\n               !w(:,   0,j,plane) =\n               !vhi(:, 0,j,plane) =" % (a, b))
                        if nv:
                            out.append("\n               !Yv(:,  0,j,plane) =")
                        out.append("\n               !w(:,  -1,j,plane) =\n               !vhi(:,-1,j,plane) =")
                        if nv:
                            out.append("\n               !Yv(:, -1,j,plane) =")
                        out.append("\n            end do\n         end if\n")
                if hi:
                    out.append("\n         if(gx(plane) .eq. ngx(plane)) then\n            !i=ni+1/2")
                    for a, b in hi:
                        out.append("\n            do j=max(%5i,nys(plane)),min(nye(plane),%5i)"
                                   "\n               !w(:,  ni(plane)+1,j,plane) =\n               !vhi(:,ni(plane)+1,j,plane) ="
                                   % (a, b))
                        if nv:
                            out.append("\n               !Yv(:, ni(plane)+1,j,plane) =")
                        out.append("\n               !w(:,  ni(plane)+2,j,plane) =\n               !vhi(:,ni(plane)+2,j,plane) =")
                        if nv:
                            out.append("\n               !Yv(:, ni(plane)+2,j,plane) =")
                        out.append("\n            end do\n         end if")
            else:
                if lo:
                    out.append("\n         if(gy(plane) .eq. 1) then\n            !j=1/2")
                    for a, b in lo:
                        out.append("\n            do i=max(%5i,nxs(plane)),min(nxe(plane),%5i)"
                                   "\n               !w(:,  i, 0,plane) =\n               !vhi(:,i, 0,plane) =" % (a, b))
                        if nv:
                            out.append("\n               !Yv(:, i, 0,plane) =")
                        out.append("\n               !w(:,  i,-1,plane) =\n               !vhi(:,i,-1,plane) =")
                        if nv:
                            out.append("\n               !Yv(:, i,-1,plane) =")
                        out.append("\n            end do\n         end if\n")
                if hi:
                    out.append("\n         if(gy(plane) .eq.  ngy(plane)) then\n            !j=nj+1/2")
                    for a, b in hi:
                        out.append("\n            do i=max(%5i,nxs(plane)),min(nxe(plane),%5i)"
                                   "\n               !w(:,  i,nj(plane)+1,plane) =\n               !vhi(:,i,nj(plane)+1,plane) ="
                                   % (a, b))
                        if nv:
                            out.append("\n               !Yv(:, i,nj(plane)+1,plane) =")
                        out.append("\n               !w(:,  i,nj(plane)+2,plane) =\n               !vhi(:,i,nj(plane)+2,plane) =")
                        if nv:
                            out.append("\n               !Yv(:, i,nj(plane)+2,plane) =")
                        out.append("\n            end do\n         end if")
        if direction == "i":
            out.append("\n      end select\n   end do\n\n   call MPI_COMMUNICATIONS_I_DIRECTION\n")
        else:
            out.append("\n      end select\n   end do\n\n   call MPI_COMMUNICATIONS_J_DIRECTION\n\n   call set_corners\n")
    out.append(g.take("condition.tail.f90"))
    with open(g.path("condition.raw.f90"), "w") as fh:
        fh.write("".join(out))


def gen_cond(g, grid_path, aboutnv):
    """store/cond/core/gen_cond.py for a single process (personal computer and
    GPU architectures): the block connectivity records of cut_copro000.inp
    and condition.raw.f90.  No MPI communication files exist with one
    process (out_MPI writes none, MaxMPIcomm = 0)."""
    planes = F.read_plot3d(grid_path)
    recs, tsm = F.connectivity(planes)
    if recs:
        with open(g.path("cut_copro000.inp"), "w") as fh:
            fh.write(F.format_cut_copro(recs, 0))
    out_cond(g, tsm, 0, aboutnv)
    for name in ("fetchMPI.py", "mod_cond.py", "out_cond.py", "read_plot3d.py", "set_cond_var.py", "gen_cond.py"):
        if os.path.exists(g.path(name)):
            os.remove(g.path(name))
    return tsm


SIDES = ("SCFD_SIDE_ILO", "SCFD_SIDE_IHI", "SCFD_SIDE_JLO", "SCFD_SIDE_JHI")


def gpu_files(g, sel, tsm, val_dt):
    """The GPU architecture's generated files: scfd_gpu_driver.f90 with the
    selections of checkout.inp, scfd_gpu_chem.f90 for the thermal model, and
    scfd_gpu_bc.raw.f90, the boundary-descriptor template the user completes
    into scfd_gpu_bc.f90 as condition.raw.f90 is completed into condition.f90."""
    muscl = sel["recon"] == 1
    fromto = [("GPU_MUSCL_USE", "use half_value, only: phi_mus, k_mus" if muscl else ""),
              ("GPU_DIM", "0" if sel["dimension"] == "2d" else "1"),
              ("GPU_DT_MODE", str(val_dt)),
              ("GPU_SCHEME", str(sel["time_scheme"])),
              ("GPU_RECON", str(sel["recon"])),
              ("GPU_VISCOUS", str(sel["viscous"])),
              ("GPU_THERMO", str(sel["thermal_model"])),
              ("GPU_PHI", "phi_mus" if muscl else "0d0"),
              ("GPU_KAPPA", "1.4d0"), ("GPU_RGAS", "287d0"), ("GPU_NU", "1.6d-5"),
              ("GPU_K", "k_mus" if muscl else "0d0")]
    g.raw2pro("scfd_gpu_driver.raw.f90", "scfd_gpu_driver.f90", fromto)
    keep = "scfd_gpu_chem.chemkin.f90" if sel["thermal_model"] in (1, 2) else "scfd_gpu_chem.none.f90"
    for name in ("scfd_gpu_chem.chemkin.f90", "scfd_gpu_chem.none.f90"):
        if name == keep:
            os.replace(g.path(name), g.path("scfd_gpu_chem.f90"))
        else:
            os.remove(g.path(name))
    ranges = []
    for p, sides in enumerate(tsm):
        for cind in range(2):
            for lu in range(2):
                for a, b in sides[cind][lu]:
                    ranges.append((p + 1, SIDES[2 * cind + lu], a, b))
    lines = ["! Boundary descriptors of this case for scfd_set_bc: one per side range that",
             "! no block interface covers (the ranges of condition.raw.f90).  Every entry",
             "! starts as zero gradient (SCFD_BC_EXTRAP); set kind and value(:) to what the",
             "! matching lines of condition.f90 write into the ghost cells (the SCFD_BC_*",
             "! kinds of include/scfd_b200.h), then save this file as scfd_gpu_bc.f90.",
             "module scfd_gpu_bc",
             "   use iso_c_binding",
             "   use scfd_b200_iface",
             "   implicit none",
             "contains",
             "   subroutine scfd_gpu_bc_set(ctx)",
             "      type(c_ptr),intent(in)::ctx"]
    if ranges:
        lines += ["      type(scfd_bc)::b(%d)" % len(ranges),
                  "      integer(c_int)::ierr"]
        for k, (p, side, a, b) in enumerate(ranges):
            lines.append("      b(%d) = scfd_bc(%d, %s, %d, %d, SCFD_BC_EXTRAP, 0, 0d0)" % (k + 1, p, side, a, b))
        lines += ["      ierr = scfd_set_bc(ctx, b, %d)" % len(ranges),
                  "      if(ierr .ne. 0) then",
                  "         print *,\"Error: scfd_set_bc returned status \",ierr",
                  "         stop",
                  "      end if"]
    lines += ["   end subroutine scfd_gpu_bc_set", "end module scfd_gpu_bc", ""]
    with open(g.path("scfd_gpu_bc.raw.f90"), "w") as fh:
        fh.write("\n".join(lines))


# ---- store/checkout/checkout_flow.py ---------------------------------------
def checkout_flow(root=".", inp="checkout.inp", log=print):
    """Generate <root>/checkout from <root>/checkout.inp; returns a dict of the
    selections made."""
    g = Generator(root, log=log)
    if os.path.exists(g.out):
        # the reference keeps the user's condition.f90, control.inp and grid
        # files of the previous checkout beside it (checkout_flow.py:7-18)
        for name, bak in (("condition.f90", "condition.bak.f90"), ("control.inp", "control.bak.inp")):
            if os.path.exists(g.path(name)):
                shutil.copyfile(g.path(name), os.path.join(g.root, bak))
        if os.path.isdir(g.path("grid")):
            os.makedirs(os.path.join(g.root, "grid_bak"), exist_ok=True)
            for name in os.listdir(g.path("grid")):
                shutil.copyfile(os.path.join(g.path("grid"), name), os.path.join(g.root, "grid_bak", name))
        shutil.rmtree(g.out)
    os.makedirs(g.path("grid"))
    os.makedirs(g.path("result"))
    sel = {}
    with open(os.path.join(g.root, inp)) as fp:
        g.engage("core")
        # grid file: plane count and node counts (checkout_flow.py:44-64)
        gridname = read_control_next(fp)
        gpath = os.path.join(g.root, gridname)
        with open(gpath) as fh:
            nplane = int(fh.readline().split()[-1])
            nijk = []
            for _ in range(nplane):
                a = [int(x) - 1 for x in fh.readline().split()[:3]]
                if a[2] != 0:
                    raise CheckoutError("This program cannot be applied yet to 3D problem.")
                nijk.append(a[:2])
        shutil.copyfile(gpath, os.path.join(g.path("grid"), os.path.basename(gridname)))

        log("***architecture***")
        arc = read_control_next(fp)
        if arc.upper() == "GPU":
            log("\tB200 GPU (libscfd_b200) is selected.")
            g.engage("architecture/PC")
            g.engage("architecture/GPU", store=GPU_STORE)
            sel["architecture"] = "GPU"
        else:
            try:
                val = int(arc)
            except ValueError:
                raise CheckoutError("Odd Input at architecture! value is %s" % arc) from None
            if val == 0:
                log("\tPersonal Computer is selected.")
                g.engage("architecture/PC")
                sel["architecture"] = "PC"
            elif val < 0:
                log("\tV-System[Super Computer] is selected.")
                g.engage("architecture/VC")
                sel["architecture"] = "VC"
            else:
                raise CheckoutError("the M-System architecture (MPI processes, value > 0) is not ported; use the "
                                    "reference's own generator for it")

        log("***dimension***")
        val = read_control_next_int(fp, "dimension")
        if val not in (0, 1):
            raise CheckoutError("Odd Input at dimension! value is %d" % val)
        dimension = "2d" if val == 0 else "q2d"
        g.engage("dim/" + dimension)
        sel["dimension"] = dimension

        log("***time scale***")
        val_dt = read_control_next_int(fp, "time step")
        if val_dt not in (0, 1):
            raise CheckoutError("Odd Input at time step! value is %d" % val_dt)
        g.engage("time_step/" + ("global" if val_dt == 0 else "local"))
        dt_text = "dt_grbl" if val_dt == 0 else "dt_mat(i,j,plane)"
        sel["time_step"] = "global" if val_dt == 0 else "local"

        log("***time scheme***")
        val = read_control_next_int(fp, "time scheme")
        schemes = {0: ("time_scheme/euler", "time_euler_viscous"), 1: ("time_scheme/RK2", "time_RK2_viscous"),
                   2: ("time_scheme/LU-SGS/" + dimension, "sch_lusgs"), 3: ("time_scheme/NR/" + dimension, "sch_NR"),
                   4: ("time_scheme/precon/" + dimension, "sch_precon"),
                   5: ("time_scheme/dual/" + dimension, "sch_dual"),
                   6: ("time_scheme/preconLU-SGS/" + dimension, "sch_precon")}
        if val not in schemes:
            raise CheckoutError("Odd Input at time scheme! value is %d" % val)
        if val == 5 and dimension == "q2d":
            raise CheckoutError("ERROR: This scheme cannot be used at axi-symmetric problem now.")
        if val == 5 and val_dt == 1:
            raise CheckoutError("ERROR: This scheme cannot be used at local time step.")
        if val in (4, 6) and val_dt == 0:
            raise CheckoutError("ERROR: This scheme cannot be used at global time step.")
        place, stem = schemes[val]
        g.engage(place)
        g.raw2pro(stem + ".raw.f90", stem + ".f90", [("DT_LOCAL_GLOBAL", dt_text)])
        sel["time_scheme"] = val

        log("***high order scheme***")
        val = read_control_next_int(fp, "high order scheme")
        if val not in (0, 1):
            raise CheckoutError("Odd Input at high order scheme! value is %d" % val)
        g.engage("high_order/" + ("upwind" if val == 0 else "muscl"))
        recon = val

        log("***viscosity***")
        val_vis = read_control_next_int(fp, "viscosity")
        if val_vis not in (0, 1):
            raise CheckoutError("Odd Input at viscosity! value is %d" % val_vis)

        log("***thermal model***")
        val = read_control_next_int(fp, "thermal model")
        sel["thermal_model"] = val
        if val == 0:
            g.engage("therm_lib/ideal")
            aboutnv, nv, ny = "no-nV", 1, 1
            g.raw2pro("thermal_model.raw.f90", "thermal_model.f90",
                      [("KAPPA", "1.4d0"), ("RGAS", "287d0"), ("NU", "1.6d-5")])
        elif val in (1, 2):
            g.engage("therm_lib/chemkin/core")
            g.engage("therm_lib/chemkin/uvhp/uv")
            if val == 1:
                g.engage("therm_lib/chemkin/flow/cold")
                cold = ".true."
            else:
                if val_dt == 1:
                    raise CheckoutError("Error : Chemical Kinetics Model cannot be used at local time step.")
                g.engage("therm_lib/chemkin/flow/reactive")
                cold = ".false."
            ne, ns, nr = _chem_counts(g)
            g.raw2pro("mod_chem.raw.f90", "mod_chem.f90",
                      [("ISCOLDFLOW", cold), ("NE", str(ne)), ("NS", str(ns)), ("NR", str(max(nr, 1)))])
            aboutnv, nv, ny = "no-nV", ns, ns
        elif val in (3, 4, 5):
            g.engage("therm_lib/NASA/core")
            g.engage({3: "therm_lib/NASA/flame_sheet/flow", 4: "therm_lib/NASA/cea/flow", 5: "therm_lib/NASA/cold"}[val])
            ne, ns, _ = _chem_counts(g)
            g.raw2pro("mod_chem.raw.f90", "mod_chem.f90", [("NE", str(ne)), ("NS", str(ns))])
            ny = 2
            nv = {3: 3, 4: ns, 5: 2}[val]
            aboutnv = "no-nV" if val == 5 else "with-nV"
        else:
            raise CheckoutError("Odd Input at thermal model! value is %d" % val)

    if sel["architecture"] == "GPU":
        if sel["time_scheme"] == 1:
            raise CheckoutError("the GPU architecture has no two-step Runge-Kutta (time scheme 1)")
        if sel["thermal_model"] not in (0, 1, 2):
            raise CheckoutError("the GPU architecture takes the ideal-gas and Chemkin thermal models (0-2)")
    sel.update(viscous=val_vis, recon=recon)
    if val_vis == 0:
        g.engage("viscosity/non-viscous")
    else:
        g.engage("viscosity/viscous/%s/%s" % (aboutnv, dimension))

    log("***generation of condition.raw.f90***")
    g.engage("cond/core")
    g.engage("cond/" + aboutnv)
    tsm = gen_cond(g, gpath, aboutnv)
    if sel["architecture"] == "GPU":
        gpu_files(g, sel, tsm, val_dt)

    # control.raw.inp, n_grid.f90, Makefile, main.f90 (checkout_flow.py:340-398)
    with open(g.path("control.raw.inp"), "w") as fh:
        fh.write(g.parts["control.part.inp"])
    g.raw2pro("n_grid.raw.f90", "n_grid.f90",
              [("NPLANE", str(nplane)), ("NumI", ",".join(str(a[0]) for a in nijk)),
               ("NumJ", ",".join(str(a[1]) for a in nijk)), ("NIMAX", str(max(a[0] for a in nijk))),
               ("NJMAX", str(max(a[1] for a in nijk))), ("NumY", str(ny)), ("NV", str(nv)),
               ("GridFileName", os.path.basename(gridname))])
    with open(g.path("Makefile"), "w") as fh:
        g.append(fh, "Makefile.head")
        fh.write(g.parts["Makefile.var"])
        fh.write(g.parts["Makefile.main"])
        g.append(fh, "Makefile.foot")
    top, init = g.parts["main.part_top.f90"], g.parts["main.part_init.f90"]
    pi, prim, pmain = (g.parts["main.part_point_implicit.f90"], g.parts["main.part_primitive.f90"],
                       g.parts["main.part_main.f90"])
    fromto = [("part_top\n", top), ("part_init\n", init), ("part_point_implicit\n", pi),
              ("part_primitive\n", prim), ("part_main\n", pmain)]
    with open(g.path("main.f90"), "w") as fh:
        fh.write(top)
        g.append(fh, "main.head.f90")
        fh.write(g.parts["main.part_variable.f90"])
        fh.write(init)
        g.raw2pro("main.body.raw.f90", "main.body.f90", fromto)
        g.append(fh, "main.body.f90")
        if sel["architecture"] == "GPU":
            # the GPU time-loop body replaces the scheme's own
            for name in ("main.main.raw.f90", "main.main.point_implicit.f90"):
                if os.path.exists(g.path(name)):
                    os.remove(g.path(name))
            g.raw2pro("main.main.gpu.f90", "main.main.f90", fromto)
        elif pi == "":
            g.raw2pro("main.main.raw.f90", "main.main.f90", fromto)
            if os.path.exists(g.path("main.main.point_implicit.f90")):
                os.remove(g.path("main.main.point_implicit.f90"))
        else:
            if not os.path.exists(g.path("main.main.point_implicit.f90")):
                log("This time scheme cannnot be applied to point implicit scheme.")
            g.raw2pro("main.main.point_implicit.f90", "main.main.f90", fromto)
            os.remove(g.path("main.main.raw.f90"))
        g.append(fh, "main.main.f90")
        g.append(fh, "main.foot.f90")
    for name in os.listdir(g.out):
        if name == "__init__.py" or name.endswith(".pyc"):
            os.remove(g.path(name))
    sel.update(nplane=nplane, nijk=nijk, ny=ny, nv=nv, aboutnv=aboutnv)
    return sel


def _chem_counts(g):
    """store/checkout/ckinterp.py: element, species and reaction counts of
    chem.inp (copied into the checkout as the reference does)."""
    src = os.path.join(g.root, "chem.inp")
    if not os.path.exists(src):
        raise CheckoutError("ERROR:Can't find 'chem.inp'. Please try again.")
    shutil.copyfile(src, g.path("chem.inp"))
    return ckinterp(open(src).read())


def ckinterp(text):
    """store/checkout/ckinterp.py: element, species and reaction counts of a
    chem.inp, read as the reference reads it: blocks in the order elements,
    species, thermo, reactions, each ended by a line starting with "end";
    lines starting with "!" are skipped, and so is the line starting with the
    block's (lower-case) keyword, tokens on it included; in the reaction block
    a line holding "/" or "duplicate" continues the previous reaction and any
    other line (a blank one too) starts a new one.  Where the reference would
    read past the end of the file forever, this raises CheckoutError."""
    lines = iter(text.splitlines(keepends=True))

    def nxt():
        try:
            return next(lines)
        except StopIteration:
            raise CheckoutError("chem.inp ends inside a block") from None
    elm, spc, rct = [], [], []
    for keyword, acc in (("elements", elm), ("species", spc)):
        while True:
            line = nxt()
            if line.startswith("!") or line.startswith(keyword):
                continue
            if line.startswith("end"):
                break
            acc.extend(line.split())
    while not nxt().startswith("end"):
        pass
    while True:
        line = nxt()
        if line.startswith("!") or line.startswith("reactions"):
            continue
        if line.startswith("end"):
            break
        if "/" in line or "duplicate" in line.lower():
            rct[-1] += line
        else:
            rct.append(line)
    return len(elm), len(spc), len(rct)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--root", default=".", help="reference checkout holding store/ and checkout.inp")
    args = ap.parse_args(argv)
    if not os.path.exists(os.path.join(args.root, "checkout.inp")):
        print("You have to make input file.")
        return 1
    try:
        checkout_flow(args.root)
    except CheckoutError as e:
        print(e)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
