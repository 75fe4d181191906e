#!/usr/bin/env python3
"""Build the PaStiX reference CPU path into oracle/_ref/ (test oracle only).

Recipe (no reference build system is run):
  1. precgen.py derives the s/d/c/z (and mixed ds/zc) sources from the
     reference's z sources into oracle/_ref/gen/;
  2. gcc compiles the reference's library sources where they lie under the
     reference tree (plus the generated copies) together with the project's
     own spm stand-in (spm_standin.c) and config header;
  3. everything links into oracle/_ref/libpastix_ref.so against the
     LP64 OpenBLAS that ships with opencv-python-headless (cblas + LAPACKE
     names).

Nothing from the reference tree is copied into the repository: generated
files and objects live only under the git-ignored oracle/_ref/.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref")
GEN = os.path.join(OUT, "gen")
OBJ = os.path.join(OUT, "obj")
# the reference tree sits beside the repository (override: PASTIX_REFERENCE_ROOT)
REF = os.environ.get("PASTIX_REFERENCE_ROOT",
                     os.path.join(os.path.dirname(os.path.dirname(ORACLE)), "reference"))


def find_openblas():
    import site
    cands = []
    for sp in site.getsitepackages() + [site.getusersitepackages()]:
        cands += glob.glob(os.path.join(sp, "opencv_python_headless.libs", "libopenblas*.so"))
    if not cands:
        raise RuntimeError("LP64 OpenBLAS (opencv-python-headless bundle) not found")
    return cands[0]


NORMAL4 = "sdcz"
GENERATED = {
    # path: precisions
    "common/z_integer.c": NORMAL4,
    "bcsc/bcsc_z.h": NORMAL4,
    "bcsc/bcsc_zinit.c": NORMAL4,
    "bcsc/bcsc_znorm.c": NORMAL4,
    "bcsc/bcsc_zspmv.c": NORMAL4,
    "bcsc/bvec_zcompute.c": NORMAL4,
    "bcsc/bvec_zlapmr.c": NORMAL4,
    "bcsc/bvec_zmpi_comm.c": NORMAL4,
    "sopalin/coeftab_z.h": NORMAL4,
    "sopalin/coeftab_z.c": NORMAL4,
    "sopalin/coeftab_zinit.c": NORMAL4,
    "sopalin/sequential_zdiag.c": NORMAL4,
    "sopalin/sequential_zgetrf.c": NORMAL4,
    "sopalin/sequential_zhetrf.c": "cz",
    "sopalin/sequential_zpotrf.c": NORMAL4,
    "sopalin/sequential_zpxtrf.c": "cz",
    "sopalin/sequential_zsytrf.c": NORMAL4,
    "sopalin/sequential_ztrsm.c": NORMAL4,
    "sopalin/coeftab_zcinit.c": "zc",
    "refinement/z_refine_bicgstab.c": NORMAL4,
    "refinement/z_refine_functions.c": NORMAL4,
    "refinement/z_refine_functions.h": NORMAL4,
    "refinement/z_refine_gmres.c": NORMAL4,
    "refinement/z_refine_grad.c": NORMAL4,
    "refinement/z_refine_pivot.c": NORMAL4,
    "kernels/pastix_zcores.h": NORMAL4,
    "kernels/pastix_zcuda.h": NORMAL4,
    "kernels/pastix_zlrcores.h": NORMAL4,
    "kernels/z_nan_check.h": NORMAL4,
    "kernels/cpucblk_zpack.h": NORMAL4,
    "kernels/pastix_zccores.h": "zc",
    "kernels/cpucblk_zcinit.c": "zc",
}
for k in ["core_zgemdm", "core_zgetmo", "core_zgeadd", "core_zplrnt", "core_ztradd",
          "core_zgemmsp", "core_ztrsmsp", "core_zscalo", "core_zsytrfsp", "core_zpotrfsp",
          "core_zgetrfsp", "core_zlrnrm", "core_zlrdbg", "core_zlr2xx", "core_zxx2lr",
          "core_zxx2fr", "core_zlrmm", "core_zpqrcp", "core_zrqrcp", "core_ztqrcp",
          "core_zrqrrt", "core_zlrothu", "core_zgelrops_svd", "core_zgelrops",
          "cpucblk_zinit", "cpucblk_zcompress", "cpucblk_zdiff", "cpucblk_zadd",
          "cpucblk_zschur", "cpucblk_zmpi_coeftab", "cpucblk_zmpi_rhs_fwd",
          "cpucblk_zmpi_rhs_bwd", "cpucblk_zpack", "solve_ztrsmsp"]:
    GENERATED["kernels/%s.c" % k] = NORMAL4
GENERATED["kernels/core_zhetrfsp.c"] = "cz"
GENERATED["kernels/core_zpxtrfsp.c"] = "cz"

PLAIN = """graph/graph.c graph/graph_compute_projection.c graph/graph_connected_components.c
graph/graph_io.c graph/graph_isolate.c graph/graph_prepare.c
order/order.c order/order_add_isolate.c order/order_amalgamate.c order/order_apply_level_order.c
order/order_check.c order/order_compute_personal.c order/order_find_supernodes.c order/order_grids.c
order/order_io.c order/pastix_subtask_order.c
symbol/fax_csr.c symbol/fax_csr_amalgamate.c symbol/fax_csr_direct.c symbol/fax_csr_iluk.c
symbol/symbol.c symbol/symbol_base.c symbol/symbol_check.c symbol/symbol_cost.c
symbol/symbol_cost_flops.c symbol/symbol_cost_perfs.c symbol/symbol_draw.c symbol/symbol_draw_map.c
symbol/symbol_fax_direct.c symbol/symbol_fax_iluk.c symbol/symbol_io.c symbol/symbol_reordering.c
symbol/symbol_expand.c symbol/symbol_reorder.c
symbol/pastix_subtask_reordering.c symbol/pastix_subtask_symbfact.c
blend/pastix_subtask_blend.c blend/pastix_task_analyze.c blend/blendctrl.c blend/cand.c
blend/cand_gendot.c blend/cost.c blend/elimintree.c blend/extendVector.c blend/extracblk.c
blend/propmap.c blend/simu.c blend/simu_run.c blend/simu_task.c blend/solver.c
blend/solver_backup.c blend/solver_check.c blend/solver_copy.c blend/solver_draw.c
blend/solver_io.c blend/solver_matrix_gen.c blend/solver_matrix_gen_utils.c blend/solver_recv.c
blend/splitsymbol.c
common/api.c common/integer.c common/isched.c common/models.c common/get_options.c
common/parse_options.c common/check_options.c common/getline.c common/isched_nohwloc.c
bcsc/bcsc.c bcsc/bvec.c
sopalin/coeftab.c sopalin/schur.c sopalin/diag.c sopalin/pastix_task_sopalin.c
sopalin/pastix_task_solve.c sopalin/pastix.c sopalin/pastix_rhs.c
refinement/pastix_task_refine.c
kernels/kernels.c kernels/kernels_trace.c kernels/lowrank.c kernels/queue.c""".split()


def gen_outputs():
    outs = []
    for path, precs in GENERATED.items():
        if not path.endswith(".c"):
            continue
        d, b = os.path.split(path)
        if precs == "zc":
            outs.append((os.path.join(GEN, d, b.replace("zc", "ds", 1)), "ds"))
            outs.append((os.path.join(REF, path), "zc"))
            continue
        for p in precs:
            if p == "z":
                outs.append((os.path.join(REF, path), "z"))
            else:
                sys.path.insert(0, HERE)
                import precgen
                outs.append((os.path.join(GEN, d, precgen.out_name(b, p)), p))
    return outs


def includes():
    inc = [HERE, GEN]
    for sub in ("kernels", "common", "refinement", "sopalin", "bcsc"):
        inc.append(os.path.join(GEN, sub))
    inc.append(REF)
    for sub in ("include", "kernels", "common", "refinement", "sopalin", "bcsc"):
        inc.append(os.path.join(REF, sub))
    return ["-I" + i for i in inc]


CFLAGS = ["-O2", "-fPIC", "-std=gnu11", "-w", "-fno-strict-aliasing", "-pthread",
          "-DNDEBUG"]


def compile_one(args):
    src, prec, obj = args
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(f) for f in
                  glob.glob(os.path.join(HERE, "*.[ch]")) + glob.glob(os.path.join(HERE, "pastix", "*.h"))])
    if os.path.exists(obj) and os.path.getmtime(obj) > newest:
        return obj, None
    flags = list(CFLAGS)
    if prec:
        flags.append("-DPRECISION_%s" % prec)
    cmd = ["gcc"] + flags + includes() + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr
    return obj, None


# The reference's unblocked LDL^h kernel (kernels/core_zhetrfsp.c:91-92
# core_zhetf2sp) copies column k of the diagonal block into row k with
# cblas_zcopy(m, Amk, 1, Akm, lda) and then conjugates it with
# LAPACKE_zlacgv_work(m, Akm, 1): increment 1 instead of lda, so it
# conjugates m entries of column k+1 (the new diagonal and the lower
# entries below it) instead of row k.  For a Hermitian matrix with non-real
# off-diagonal entries the factors are then not those of A (real-valued
# Hermitian matrices are unaffected).  libpastix_ref_hefix.so is the same
# build with that one increment set to lda (in generated copies under
# oracle/_ref/gen/hefix/), used to pin the GPU LDL^h on complex data.
HEFIX = [("kernels/core_zhetrfsp.c", "z", "LAPACKE_zlacgv_work( m, Akm, 1 )", "LAPACKE_zlacgv_work( m, Akm, lda )"),
         ("kernels/core_chetrfsp.c", "c", "LAPACKE_clacgv_work( m, Akm, 1 )", "LAPACKE_clacgv_work( m, Akm, lda )")]


def build_hefix(units, blas):
    fixdir = os.path.join(GEN, "hefix", "kernels")
    os.makedirs(fixdir, exist_ok=True)
    repl = {}
    for rel, prec, old, new in HEFIX:
        src = os.path.join(REF if prec == "z" else GEN, rel)
        text = open(src).read()
        if text.count(old) != 1:
            raise RuntimeError("hefix: pattern not found once in %s" % src)
        dst = os.path.join(fixdir, os.path.basename(rel))
        with open(dst, "w") as f:
            f.write(text.replace(old, new))
        obj = os.path.join(OBJ, "hefix__" + os.path.basename(rel) + "." + prec + ".o")
        o, err = compile_one((dst, prec, obj))
        if err:
            raise RuntimeError(err)
        repl[src] = obj
    objs = [repl.get(u[0], u[2]) for u in units]
    if len([u for u in units if u[0] in repl]) != len(HEFIX):
        raise RuntimeError("hefix: kernels not found among the compiled units")
    so = os.path.join(OUT, "libpastix_ref_hefix.so")
    subprocess.check_call(["gcc", "-shared", "-o", so] + objs +
                          [blas, "-Wl,-Bsymbolic", "-Wl,--disable-new-dtags", "-Wl,-rpath," + os.path.dirname(blas),
                           "-lm", "-pthread"])


# Second build of the reference sources with the GPU layer plugged in
# (pastix_b200/refplug/pastix_gpu_plug.c): the same objects, the plug, and
# one --wrap per plug point, linked against pastix_b200/lib/libpastix_gpu.so.
# The reference's own public API then factorizes, solves and refines on the
# GPU (tests/test_dropin.py runs example/simple.c's call sequence on it).
REPO = os.path.dirname(ORACLE)
PLUG_SRC = os.path.join(REPO, "pastix_b200", "refplug", "pastix_gpu_plug.c")
GPU_LIBDIR = os.path.join(REPO, "pastix_b200", "lib")
PLUG_WRAPS = (["coeftabInit", "pastixFinalize"] +
              ["sopalin_%s%s" % (p, f) for p in "sdcz" for f in ("potrf", "getrf", "sytrf", "trsm", "diag")] +
              ["sopalin_chetrf", "sopalin_zhetrf"] +
              ["%s_%s_smp" % (p, f) for p in "dz" for f in ("grad", "gmres")])


def build_gpuplug(units, blas):
    if not os.path.exists(os.path.join(GPU_LIBDIR, "libpastix_gpu.so")):
        print("libpastix_gpu.so not built; skipping the GPU-plugged reference build")
        return
    obj = os.path.join(OBJ, "pastix_gpu_plug.o")
    cmd = ["gcc"] + CFLAGS + includes() + ["-I" + os.path.join(REPO, "include"), "-c", PLUG_SRC, "-o", obj]
    subprocess.check_call(cmd)
    so = os.path.join(OUT, "libpastix_gpuplug.so")
    wraps = ["-Wl,--wrap=" + w for w in PLUG_WRAPS]
    subprocess.check_call(["gcc", "-shared", "-o", so] + [u[2] for u in units] + [obj] + wraps +
                          ["-L" + GPU_LIBDIR, "-lpastix_gpu",
                           "-Wl,-rpath,$ORIGIN/../../pastix_b200/lib", blas, "-Wl,-Bsymbolic",
                           "-Wl,--disable-new-dtags", "-Wl,-rpath," + os.path.dirname(blas), "-lm", "-pthread"])


def main():
    if not os.path.isdir(REF):
        print("reference tree not present; skipping the reference build")
        return 0
    os.makedirs(GEN, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    jobs = ["%s:%s" % (p, "ds" if v == "zc" else v.replace("z", "")) for p, v in GENERATED.items()]
    jobs = [j for j in jobs if not j.endswith(":")]
    subprocess.check_call([sys.executable, os.path.join(HERE, "precgen.py"), REF, GEN] + jobs)

    units = []
    for src, prec in gen_outputs():
        rel = os.path.relpath(src, GEN if src.startswith(GEN) else REF)
        units.append((src, prec, os.path.join(OBJ, rel.replace("/", "__") + "." + prec + ".o")))
    for p in PLAIN:
        units.append((os.path.join(REF, p), None, os.path.join(OBJ, p.replace("/", "__") + ".o")))
    units.append((os.path.join(HERE, "spm_standin.c"), None, os.path.join(OBJ, "spm_standin.o")))
    units.append((os.path.join(HERE, "ref_glue.c"), None, os.path.join(OBJ, "ref_glue.o")))

    errors = []
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for obj, err in ex.map(compile_one, units):
            if err:
                errors.append((obj, err))
    if errors:
        for obj, err in errors[:8]:
            print("== %s\n%s" % (obj, err[:3000]))
        print("%d compile errors" % len(errors))
        return 1
    blas = find_openblas()
    so = os.path.join(OUT, "libpastix_ref.so")
    objs = [u[2] for u in units]
    cmd = ["gcc", "-shared", "-o", so] + objs + [blas, "-Wl,--disable-new-dtags", "-Wl,-rpath," + os.path.dirname(blas),
                                                 "-lm", "-pthread"]
    subprocess.check_call(cmd)
    build_hefix(units, blas)
    build_gpuplug(units, blas)
    print("built", so)
    return 0


if __name__ == "__main__":
    sys.exit(main())
