"""Build recipe for the oracle (test infrastructure, never shipped).

* ``oracle/_build/liboracle.so`` -- the C restatement in ``oracle.c``
  (gcc, FP64, ``-ffp-contract=off``, OpenMP for the CPU baseline).
* ``oracle/_ref/libref_kdtree.so`` -- the reference's own ``external/kdtree/KDTree.h``
  compiled from its sources where they lie (plus ``external/timers/timer_eb.cpp`` and
  ``external/graphics_lib/utilities/Vec3d.cpp``).
* ``oracle/_ref/libref_grid.so`` -- the reference's own ``Grid::generateStencilsHash``
  (``src/grids/grid_interface.cpp``), through ``oracle/ref_grid.cpp``;
* ``oracle/_ref/libref_rbf.so`` -- the reference's own ``src/rbffd/rbfs/rbf_gaussian.h``
  and ``src/utils/geom/cart2sph.cpp``, with ``oracle/shim/armadillo`` standing in
  for the Armadillo header that ``rbf.h`` includes.
* ``oracle/_ref/libref_norms.so`` -- the reference's own ``src/utils/norms.cpp`` with
  ``PDE::calcSolNorms``' relative rule, through ``oracle/ref_norms.cpp``.
* ``oracle/_ref/libref_mmio.so`` -- the reference's own ``external/nist/mmio.cpp``
  (the Matrix Market header of its weight files).

* ``oracle/_ref/libref_rbffd.so`` -- the reference's own hot path through
  ``oracle/ref_rbffd.cpp``: ``src/rbffd/rbffd.cpp`` (weights, getStencilLHS/RHS,
  applyWeightsForDeriv), ``src/pdes/{pde,time_dependent_pde}.cpp`` (RK4),
  ``src/pdes/hyperbolic/{cosine_bell,vortex_rollup}.cpp``, ``src/grids/{grid_interface,
  domain}.cpp`` and their utilities, unmodified, against ``oracle/shim/armadillo``
  (dense matrices; ``arma::solve`` as partial-pivot LU) and ``oracle/shim/mpi.h``
  (one rank).  ``oracle.c`` is checked against it bit for bit.

The ``_ref`` libraries are built only where the reference tree exists and
travel prebuilt elsewhere.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: RBFFD_REFERENCE_ROOT if set, else a directory named
# "reference" beside the repository's own directory.  Where neither exists the
# reference pieces are skipped (their prebuilt libraries are used as they are).
REF = os.environ.get("RBFFD_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


# The reference's hot path compiled as a whole (oracle/ref_rbffd.cpp): RBFFD,
# PDE / TimeDependentPDE, CosineBell, VortexRollup and what they need.
REF_CORE_SOURCES = [
    "src/rbffd/rbffd.cpp", "src/grids/grid_interface.cpp", "src/grids/domain.cpp", "src/pdes/pde.cpp",
    "src/pdes/time_dependent_pde.cpp", "src/pdes/hyperbolic/cosine_bell.cpp", "src/pdes/hyperbolic/vortex_rollup.cpp",
    "src/utils/comm/communicator.cpp", "src/utils/comm/mpisendable.cpp", "src/utils/norms.cpp", "src/utils/random.cpp",
    "src/utils/geom/cart2sph.cpp", "external/nist/mmio.cpp", "external/timers/timer_eb.cpp",
    "external/graphics_lib/utilities/Vec3d.cpp", "external/graphics_lib/utilities/CVec3.cpp",
    "external/graphics_lib/utilities/Vec3i.cpp",
]


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed: " + " ".join(cmd))


def build_oracle(force=False):
    out = os.path.join(HERE, "_build", "liboracle.so")
    src = os.path.join(HERE, "oracle.c")
    if force or _newer(out, [src]):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        _run(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c11",
              src, "-o", out, "-lm"])
    return out


def build_ref(force=False):
    """Compile the reference pieces; returns the list of built paths ([] if no reference tree)."""
    if not os.path.isdir(os.path.join(REF, "external", "kdtree")):
        return []
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    util = os.path.join(REF, "external", "graphics_lib", "utilities")
    # KDTree's MyHeaps.h uses dynamic exception specifications, so it needs
    # C++98; the RBF header builds with the compiler's default standard, where
    # pow(double, int) is pow(double, double) as in C (under C++98 libstdc++
    # would use repeated multiplication instead, a 1-ulp difference in HV).
    common = ["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-w",
              "-DUSE_DOUBLE_VEC3", "-include", "ctime", "-include", "cstdio"]
    built = []
    kd = os.path.join(outdir, "libref_kdtree.so")
    kd_src = [os.path.join(HERE, "ref_kdtree.cpp"), os.path.join(REF, "external/kdtree/KDTree.h"),
              os.path.join(REF, "external/kdtree/MyHeaps.h")]
    if force or _newer(kd, kd_src):
        _run(common + ["-std=c++98", "-I" + os.path.join(REF, "external/kdtree"), "-I" + os.path.join(REF, "external/timers"),
                       "-I" + util, kd_src[0], os.path.join(REF, "external/timers/timer_eb.cpp"),
                       os.path.join(util, "Vec3d.cpp"), "-o", kd])
    built.append(kd)
    rb = os.path.join(outdir, "libref_rbf.so")
    rb_src = [os.path.join(HERE, "ref_rbf.cpp"), os.path.join(REF, "src/rbffd/rbfs/rbf_gaussian.h"),
              os.path.join(REF, "src/utils/geom/cart2sph.cpp")]
    if force or _newer(rb, rb_src):
        _run(common + ["-I" + os.path.join(HERE, "shim"), "-I" + os.path.join(REF, "src/rbffd"),
                       "-I" + os.path.join(REF, "src"), "-I" + util, rb_src[0], rb_src[2],
                       os.path.join(util, "Vec3d.cpp"), os.path.join(util, "CVec3.cpp"), "-o", rb])
    built.append(rb)
    gr = os.path.join(outdir, "libref_grid.so")
    gr_src = [os.path.join(HERE, "ref_grid.cpp"), os.path.join(REF, "src/grids/grid_interface.cpp"),
              os.path.join(REF, "src/grids/grid_interface.h")]
    if force or _newer(gr, gr_src):
        _run(common + ["-std=c++98"] + ["-I" + os.path.join(REF, d) for d in
                                        ("src", "src/grids", "src/utils", "external/kdtree", "external/timers",
                                         "external/nist")] +
             ["-I" + util, gr_src[0], gr_src[1], os.path.join(REF, "src/utils/random.cpp"),
              os.path.join(util, "Vec3d.cpp"), os.path.join(REF, "external/nist/mmio.cpp"),
              os.path.join(REF, "external/timers/timer_eb.cpp"), "-o", gr])
    built.append(gr)
    nm = os.path.join(outdir, "libref_norms.so")
    nm_src = [os.path.join(HERE, "ref_norms.cpp"), os.path.join(REF, "src/utils/norms.cpp")]
    if force or _newer(nm, nm_src):
        _run(common + ["-I" + os.path.join(REF, "src"), "-I" + os.path.join(REF, "src/utils"), "-I" + util,
                       nm_src[0], nm_src[1], os.path.join(REF, "src/utils/random.cpp"), os.path.join(util, "Vec3d.cpp"),
                       "-o", nm])
    built.append(nm)
    rb2 = os.path.join(outdir, "libref_rbffd.so")
    rb2_src = [os.path.join(HERE, "ref_rbffd.cpp")] + [os.path.join(REF, f) for f in REF_CORE_SOURCES]
    if force or _newer(rb2, rb2_src + [os.path.join(HERE, "shim", "armadillo"), os.path.join(HERE, "shim", "mpi.h")]):
        # The reference's own flags (CMakeLists.txt:130-140, common/LINUX_CONFIG.cmake:23): g++ -O3
        # -ftree-vectorize for x86-64 with no -march, so no FMA contraction.  Two additions: -std=gnu++14
        # (its headers use dynamic exception specifications, removed in C++17, and it needs the C++11
        # pow(double, int) its tests were pinned with), and -fno-unswitch-loops: with GCC 13.3 at -O3 the
        # loop unswitching of getStencilRHS's per-node switch sends DerType HV to the default branch
        # ("deriv type 32 is not supported yet"); the option changes no arithmetic.
        _run(["g++", "-std=gnu++14", "-O3", "-ftree-vectorize", "-fno-unswitch-loops", "-DNDEBUG", "-DUSE_KDTREE",
              "-DUSE_DOUBLE_VEC3", "-fPIC", "-shared", "-w", "-include", "ctime", "-include", "cstdio",
              "-I" + os.path.join(HERE, "shim")] +
             ["-I" + os.path.join(REF, d) for d in ("src", "src/rbffd", "src/grids", "src/utils", "src/pdes",
                                                    "external/kdtree", "external/timers", "external/nist",
                                                    "external/graphics_lib/utilities",
                                                    "tests/experiments/cosine_bell_on_sphere")] +
             rb2_src + ["-Wl,--no-undefined", "-o", rb2])
    built.append(rb2)
    mm = os.path.join(outdir, "libref_mmio.so")
    mm_src = [os.path.join(HERE, "ref_mmio.cpp"), os.path.join(REF, "external/nist/mmio.cpp")]
    if force or _newer(mm, mm_src):
        _run(["g++", "-O2", "-fPIC", "-shared", "-w", "-I" + os.path.join(REF, "external/nist")] + mm_src + ["-o", mm])
    built.append(mm)
    return built


def build(force=False):
    return [build_oracle(force)] + build_ref(force)


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv):
        print(p)
