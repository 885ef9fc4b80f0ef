"""Compile the reference's own octree / mesh / operator / transfer sources
(from the reference tree named by $DENDRO_REFERENCE, default /root/reference;
read-only) into oracle/_ref/, single-rank, against
the project-written MPI and PETSc stand-ins in oracle/ref_build/shim.

The reference at its HEAD forces Hilbert ordering inside TreeNode::operator<
(include/oct/TreeNode.txx:198-202) while its mesh layer is Morton-only; the
build therefore uses a copy of TreeNode.h / TreeNode.txx, generated into
oracle/_ref/patched/ by this script, with those five lines removed so that
the Morton comparator is used throughout.  A copy of include/hilbert/rotation.h
gets one more byte in two sprintf buffers (the Hilbert tables that every
TreeNode constructor reads overflow them by the terminator).  Nothing in the reference tree is
modified and nothing it contains is committed.

Outputs (git-ignored; they travel to the GPU box with the snapshot):
  oracle/_ref/dendro_ref       driver binary
  oracle/_ref/dendro_ref_dumpmesh  the reference's examples/src/drivers/dumpMesh.C, single rank
  oracle/_ref/stencils/*.inp   the reference's stencil tables (read from cwd)
"""
import os
import re
import shutil
import subprocess
import sys

REF = os.environ.get("DENDRO_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(HERE), "_ref")

SOURCES = [
    "src/oct/TreeNode.C", "src/oct/Construct.C", "src/oct/Balance.C", "src/oct/Coarsen.C",
    "src/oct/OctFunctions.C", "src/oct/pickBdy.C", "src/oct/BlockPart.C", "src/oct/TreeNodePointer.C",
    "src/oda/oda.C", "src/oda/odaUtils.C", "src/oda/odaPartition.C", "src/oda/private/odaFactory.C",
    "src/oda/private/odaBuildNlist.C", "src/par/parUtils.C", "src/binOps/binUtils.C", "src/point/Point.C",
    "src/hilbert/morton.cpp", "src/hilbert/sfc.cpp", "src/hilbert/hilbert.cpp", "src/hilbert/rotation.cpp",
    "src/omg/RestrictMatVec.C", "src/omg/ProlongMatVec.C", "src/omg/VtxMaps.C", "src/omg/RmatType1StencilsAux.C",
    "src/omg/RmatType2StencilsAux.C", "src/omg/omg.C", "src/test/testUtils.C",
    "examples/src/backend/omgJac.C", "examples/src/backend/handleType2Stencils.C",
    "examples/src/backend/handleType1Stencils.C",
    "examples/src/backend/elasticityJac.C", "examples/src/backend/odaJac.C", "examples/src/backend/vecMass.C",
]
INCLUDE_DIRS = ["include", "include/oct", "include/oda", "include/omg", "include/par", "include/seq",
                "include/omp_par", "include/binOps", "include/point", "include/hilbert", "include/test",
                "include/sys", "include/fem", "include/pc", "examples/include"]


# Optimisation per source file.  With the mesh set-up built at -O2 or above
# the reference crashes inside DA_blockPartStage2 (src/oda/odaPartition.C:302,
# called from DA_FactoryPart3): odaFactory.C and odaPartition.C at -O1 are
# enough for a DA built directly, omg.C at -O1 as well for the DAs that
# DAMGCreateAndSetDA builds.  These are one-time set-up; everything else, the
# operator, diagonal and transfer loops that the CPU baselines time included,
# is built at -O3.
LOW_OPT = {"src/oda/odaPartition.C", "src/oda/private/odaFactory.C", "src/omg/omg.C"}


def opt_level(src):
    return "-O1" if src in LOW_OPT else "-O3"


def patched_headers():
    pdir = os.path.join(OUT, "patched")
    os.makedirs(pdir, exist_ok=True)
    txx = open(os.path.join(REF, "include/oct/TreeNode.txx")).read().split("\n")
    # drop the forced "#ifdef HILBERT_ORDERING / #undef / #endif / #define HILBERT_ORDERING /
    # #define USE_NCA_PROPERTY" block inside operator< (lines 198-202)
    block = [l.strip() for l in txx[197:202]]
    assert block[0].startswith("#ifdef HILBERT_ORDERING") and block[4].startswith("#define USE_NCA_PROPERTY"), block
    txx = txx[:197] + txx[202:]
    open(os.path.join(pdir, "TreeNode.txx"), "w").write("\n".join(txx))
    h = open(os.path.join(REF, "include/oct/TreeNode.h")).read()
    h = re.sub(r'#include "\.\./([a-zA-Z]+)/', lambda m: '#include "' + os.path.join(REF, "include", m.group(1)) + "/", h)
    open(os.path.join(pdir, "TreeNode.h"), "w").write(h)
    # include/hilbert/rotation.h:72-143 formats 4 (8) digits into char[4]
    # (char[8]) with sprintf, writing the terminator past the buffer; the
    # copy gives the buffers room for it (Hilbert-only code, unused here)
    r = open(os.path.join(REF, "include/hilbert/rotation.h")).read()
    n4, n8 = r.count("char str[4];"), r.count("char str[8];")
    assert n4 == 2 and n8 == 2, (n4, n8)
    r = r.replace("char str[4];", "char str[5];").replace("char str[8];", "char str[9];")
    open(os.path.join(pdir, "rotation.h"), "w").write(r)
    return pdir


def main():
    if not os.path.isdir(REF):
        print("reference tree not present; skipping the reference build")
        return 0
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    pdir = patched_headers()
    inc = ["-I" + os.path.join(HERE, "shim"), "-I" + pdir] + ["-I" + os.path.join(REF, d) for d in INCLUDE_DIRS]
    flags = ["-g", "-std=c++11", "-fopenmp", "-w", "-fpermissive", "-D__USE_PVT_DA_IN_MG__", "-D__SILENT_MODE__",
             "-include", os.path.join(pdir, "rotation.h"), "-include", os.path.join(pdir, "TreeNode.h")]
    objs, procs = [], []
    for src in SOURCES + [os.path.join(HERE, "ref_driver.cpp"), os.path.join(HERE, "dump_stubs.cpp"),
                          "examples/src/drivers/dumpMesh.C"]:
        path = src if os.path.isabs(src) else os.path.join(REF, src)
        obj = os.path.join(OUT, "obj", os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(path), os.path.getmtime(__file__),
                                                             *[os.path.getmtime(os.path.join(HERE, "shim", f))
                                                               for f in os.listdir(os.path.join(HERE, "shim"))]):
            continue
        procs.append((subprocess.Popen(["g++", opt_level(src), *flags, *inc, "-c", path, "-o", obj],
                                       stdout=subprocess.PIPE,
                                       stderr=subprocess.STDOUT), src))
    bad = []
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode:
            bad.append(src)
            sys.stderr.write(f"==== {src}\n" + out.decode()[-6000:])
    if bad:
        print("reference build failed:", bad)
        return 1
    lib_objs, driver_obj, stub_obj, dump_obj = objs[:-3], objs[-3], objs[-2], objs[-1]
    subprocess.check_call(["g++", "-fopenmp", "-rdynamic", "-o", os.path.join(OUT, "dendro_ref"), *lib_objs,
                           driver_obj])
    # the mesh dump needs the octree, mesh and support sources only
    mesh_objs = [o for o, src in zip(lib_objs, SOURCES) if src.split("/")[1] in ("oct", "oda", "par", "binOps",
                                                                                   "point", "hilbert")]
    subprocess.check_call(["g++", "-fopenmp", "-rdynamic", "-o", os.path.join(OUT, "dendro_ref_dumpmesh"),
                           *mesh_objs, stub_obj, dump_obj])
    sdir = os.path.join(OUT, "stencils")
    os.makedirs(sdir, exist_ok=True)
    for f in os.listdir(os.path.join(REF, "Stencils")):
        shutil.copy(os.path.join(REF, "Stencils", f), sdir)
    print(os.path.join(OUT, "dendro_ref"))
    return 0


if __name__ == "__main__":
    sys.exit(main())
