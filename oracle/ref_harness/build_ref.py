"""Build the reference harness: milupHPC's own CUDA sources, compiled
unmodified where they lie (the tree named by MHPC_REFERENCE, by default
/root/reference), plus ref_driver.cu, into
oracle/_ref/ref_gravity, oracle/_ref/ref_sph, oracle/_ref/ref_sph_bal and
oracle/_ref/ref_integrators (the integrator update kernels, ref_integrators.cu).

TEST INFRASTRUCTURE ONLY.  The reference selects its physics with a
parameter.h per test case (testcases/*/parameter.h, copied over
include/parameter.h before a build); here the test case's header is
pre-included (-include), so its include guard shadows include/parameter.h.
Boost.MPI, MPI and libconfig are replaced by the single-rank shims in
oracle/ref_harness/shim.  ref_sph_bal is the Sedov build with the Balsara
switch on (balsara_on.h pre-included after the test case's parameter.h).  Flags follow the reference Makefile (-dc -fmad=false
-O3), for sm_100a.  Outputs go only to oracle/_ref/ (git-ignored).
"""
import os
import subprocess
import sys

# the milupHPC source tree (read only): MHPC_REFERENCE, default /root/reference
REF = os.environ.get("MHPC_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(HERE), "_ref")

COMMON = ["src/particles.cu", "src/particle_handler.cpp", "src/subdomain_key_tree/tree.cu",
          "src/subdomain_key_tree/tree_handler.cpp", "src/subdomain_key_tree/subdomain.cu", "src/helper.cu",
          "src/helper_handler.cpp", "src/device_rhs.cu", "src/cuda_utils/cuda_utilities.cu",
          "src/cuda_utils/cuda_launcher.cu", "src/cuda_utils/cuda_runtime.cpp", "src/cuda_utils/linalg.cu",
          "src/utils/logger.cpp", "src/materials/material.cu"]
SPH_SRCS = COMMON + ["src/materials/material_handler.cpp", "src/sph/sph.cu", "src/sph/density.cu",
                     "src/sph/soundspeed.cu", "src/sph/pressure.cu", "src/sph/internal_forces.cu",
                     "src/sph/kernel.cu", "src/sph/kernel_handler.cu", "src/sph/stress.cu",
                     "src/sph/artificial_stress.cu", "src/sph/viscosity.cu"]
INTEG_SRCS = SPH_SRCS + ["src/integrator/device_leapfrog.cu", "src/integrator/device_explicit_euler.cu",
                         "src/integrator/device_predictor_corrector_euler.cu"]
# name: (test-case parameter.h, extra pre-included header of this directory or None, sources, driver)
BUILDS = {
    "gravity": ("testcases/plummer/parameter.h", None, COMMON + ["src/gravity/gravity.cu"], "ref_driver.cu"),
    "sph": ("testcases/sedov/parameter.h", None, SPH_SRCS, "ref_driver.cu"),
    "sph_bal": ("testcases/sedov/parameter.h", "balsara_on.h", SPH_SRCS, "ref_driver.cu"),
    "integrators": ("testcases/sedov/parameter.h", None, INTEG_SRCS, "ref_integrators.cu"),
}


def build(verbose=False):
    if not os.path.isdir(REF):
        return False
    for name, (param, extra, srcs, driver) in BUILDS.items():
        objdir = os.path.join(OUT, "obj_" + name)
        os.makedirs(objdir, exist_ok=True)
        exe = os.path.join(OUT, "ref_" + name)
        flags = ["nvcc", "-std=c++14", "-x", "cu", "-dc", "-w", "-fmad=false", "-O3",
                 "-gencode", "arch=compute_100a,code=sm_100a", "-include", os.path.join(REF, param)]
        if extra:
            flags += ["-include", os.path.join(HERE, extra)]
        flags += ["-I" + os.path.join(HERE, "shim"), "-I" + os.path.join(REF, "include")]
        objs = []
        for s in srcs + [os.path.join(HERE, driver)]:
            src = s if os.path.isabs(s) else os.path.join(REF, s)
            obj = os.path.join(objdir, os.path.basename(s).replace(".", "_") + ".o")
            objs.append(obj)
            if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src):
                continue
            cmd = flags + [src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
        if not os.path.exists(exe) or any(os.path.getmtime(o) > os.path.getmtime(exe) for o in objs):
            subprocess.check_call(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-o", exe] + objs)
    return True


if __name__ == "__main__":
    ok = build(verbose="-v" in sys.argv)
    print("reference harness built" if ok else "no reference tree; harness not built")
