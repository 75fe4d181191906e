#!/usr/bin/env python3
"""Precision generator for building the PaStiX reference as a test oracle.

The reference writes every numerical source once, in double-complex ("z"),
and relies on the morse_cmake precision generator (an empty submodule in the
reference tree, see .gitmodules) plus cmake_modules/local_subs.py to derive
the s/d/c copies ("@precisions normal z -> c d s") and the mixed ds copy
("@precisions mixed zc -> ds").  This script restates that step with its own
substitution table: for each target precision it rewrites type names, BLAS and
LAPACKE routine names, PaStiX's z-prefixed identifiers and the complex-only
intrinsics (conj/creal/cabs/csqrt) of the real precisions.

Outputs go to oracle/_ref/gen/ only.  Test infrastructure only.
"""
import os
import re
import sys

PRECS = "sdcz"

# --- ordered (s, d, c, z) substitution rules; the z column is a regex -------
# Types first (longest names first so that complex32 is not caught twice).
NORMAL = [
    ("float", "double", "pastix_complex32_t", r"\bpastix_complex64_t\b"),
    ("float", "float", "pastix_complex32_t", r"\bpastix_complex32_t\b"),
    ("float", "double", "spm_complex32_t", r"\bspm_complex64_t\b"),
    ("PastixFloat", "PastixDouble", "PastixComplex32", r"\bPastixComplex64\b"),
    ("PastixFloat", "PastixFloat", "PastixComplex32", r"\bPastixComplex32\b"),
    ("SpmFloat", "SpmDouble", "SpmComplex32", r"\bSpmComplex64\b"),
    ("FLT_EPSILON", "DBL_EPSILON", "FLT_EPSILON", r"\bDBL_EPSILON\b"),
    ("FLT_MAX", "DBL_MAX", "FLT_MAX", r"\bDBL_MAX\b"),
    ("MPI_FLOAT", "MPI_DOUBLE", "MPI_COMPLEX32", r"\bMPI_COMPLEX64\b"),
    ("PASTIX_MPI_FLOAT", "PASTIX_MPI_DOUBLE", "PASTIX_MPI_COMPLEX32", r"\bPASTIX_MPI_COMPLEX64\b"),
    # Transposition flavours: real precisions have no conjugate transpose.
    ("PastixTrans", "PastixTrans", "PastixConjTrans", r"\bPastixConjTrans\b"),
    ("CblasTrans", "CblasTrans", "CblasConjTrans", r"\bCblasConjTrans\b"),
    ("PastixSymmetric", "PastixSymmetric", "PastixHermitian", r"\bPastixHermitian\b"),
    # BLAS / LAPACKE routines whose real names differ.
    ("cblas_snrm2", "cblas_dnrm2", "cblas_scnrm2", r"\bcblas_dznrm2\b"),
    ("cblas_sscal", "cblas_dscal", "cblas_csscal", r"\bcblas_zdscal\b"),
    ("cblas_isamax", "cblas_idamax", "cblas_icamax", r"\bcblas_izamax\b"),
    ("cblas_ssyrk", "cblas_dsyrk", "cblas_cherk", r"\bcblas_zherk\b"),
    ("cblas_ssyr", "cblas_dsyr", "cblas_cher", r"\bcblas_zher\b"),
    ("cblas_sger", "cblas_dger", "cblas_cgeru", r"\bcblas_zgeru\b"),
    ("cblas_sger", "cblas_dger", "cblas_cgerc", r"\bcblas_zgerc\b"),
    ("cblas_ssymm", "cblas_dsymm", "cblas_chemm", r"\bcblas_zhemm\b"),
    ("LAPACKE_slansy", "LAPACKE_dlansy", "LAPACKE_clanhe", r"\bLAPACKE_zlanhe"),
    ("LAPACKE_sormqr", "LAPACKE_dormqr", "LAPACKE_cunmqr", r"\bLAPACKE_zunmqr"),
    ("LAPACKE_sormlq", "LAPACKE_dormlq", "LAPACKE_cunmlq", r"\bLAPACKE_zunmlq"),
    ("LAPACKE_sorgqr", "LAPACKE_dorgqr", "LAPACKE_cungqr", r"\bLAPACKE_zungqr"),
    ("LAPACKE_sorglq", "LAPACKE_dorglq", "LAPACKE_cunglq", r"\bLAPACKE_zunglq"),
    ("LAPACKE_slag2d", "LAPACKE_dlag2s", "LAPACKE_clag2z", r"\bLAPACKE_zlag2c"),
    ("LAPACKE_slag2d", "LAPACKE_slag2d", "LAPACKE_clag2z", r"\bLAPACKE_clag2z"),
    ("FLOPS_SORMQR", "FLOPS_DORMQR", "FLOPS_CUNMQR", r"\bFLOPS_ZUNMQR\b"),
    ("FLOPS_SORMLQ", "FLOPS_DORMLQ", "FLOPS_CUNMLQ", r"\bFLOPS_ZUNMLQ\b"),
    ("FLOPS_SORGQR", "FLOPS_DORGQR", "FLOPS_CUNGQR", r"\bFLOPS_ZUNGQR\b"),
    ("FLOPS_SSYTRF", "FLOPS_DSYTRF", "FLOPS_CHETRF", r"\bFLOPS_ZHETRF\b"),
    # The conjugated dot product is the plain one in real arithmetic.
    ("vec_sdotu", "vec_ddotu", "vec_cdotc", r"vec_zdotc"),
    # Generic BLAS / LAPACKE / flop-count prefixes.
    ("cblas_s", "cblas_d", "cblas_c", r"\bcblas_z"),
    ("LAPACKE_s", "LAPACKE_d", "LAPACKE_c", r"\bLAPACKE_z"),
    ("MYLAPACKE_s", "MYLAPACKE_d", "MYLAPACKE_c", r"\bMYLAPACKE_z"),
    ("FLOPS_S", "FLOPS_D", "FLOPS_C", r"\bFLOPS_Z"),
    ("cublasS", "cublasD", "cublasC", r"\bcublasZ"),
    # Complex intrinsics (the real precisions drop them).
    ("fabsf", "fabs", "cabsf", r"\bcabs\b"),
    ("sqrtf", "sqrt", "csqrtf", r"\bcsqrt\b"),
    ("", "", "conjf", r"\bconj\b"),
    ("", "", "crealf", r"\bcreal\b"),
    ("", "", "CBLAS_SADDR", r"\bCBLAS_SADDR\b"),
    # Constants.  (PRECISION_x guards are left alone: each generated unit is
    # compiled with -DPRECISION_<p>, so "#if defined(PRECISION_z) ||
    # defined(PRECISION_c)" selects the complex-only code.)
    ("sone", "done", "cone", r"\bzone\b"),
    ("msone", "mdone", "mcone", r"\bmzone\b"),
    ("szero", "dzero", "czero", r"\bzzero\b"),
    # PaStiX identifiers carrying the precision letter after a known prefix.
    ("core_s", "core_d", "core_c", r"core_z"),
    ("CORE_S", "CORE_D", "CORE_C", r"CORE_Z"),
    ("blok_s", "blok_d", "blok_c", r"blok_z"),
    ("cblk_s", "cblk_d", "cblk_c", r"cblk_z"),
    ("coeftab_s", "coeftab_d", "coeftab_c", r"coeftab_z"),
    ("cuda_s", "cuda_d", "cuda_c", r"cuda_z"),
    ("csc_s", "csc_d", "csc_c", r"csc_z"),
    ("pastix_s", "pastix_d", "pastix_c", r"pastix_z"),
    ("PASTIX_S", "PASTIX_D", "PASTIX_C", r"PASTIX_Z"),
    ("sequential_s", "sequential_d", "sequential_c", r"sequential_z"),
    ("thread_s", "thread_d", "thread_c", r"\bthread_z"),
    ("static_s", "static_d", "static_c", r"static_z"),
    ("dynamic_s", "dynamic_d", "dynamic_c", r"dynamic_z"),
    ("runtime_s", "runtime_d", "runtime_c", r"runtime_z"),
    ("starpu_s", "starpu_d", "starpu_c", r"starpu_z"),
    ("parsec_s", "parsec_d", "parsec_c", r"parsec_z"),
    ("sopalin_s", "sopalin_d", "sopalin_c", r"sopalin_z"),
    ("vec_s", "vec_d", "vec_c", r"vec_z"),
    ("spm_s", "spm_d", "spm_c", r"spm_z"),
    ("args_s", "args_d", "args_c", r"args_z"),
    ("solve_s", "solve_d", "solve_c", r"solve_z"),
    ("_s_", "_d_", "_c_", r"_z_"),
    ("s_", "d_", "c_", r"\bz_"),
    ("spotrf_table", "dpotrf_table", "cpotrf_table", r"\bzpotrf_table\b"),
    ("sgetrf_table", "dgetrf_table", "cgetrf_table", r"\bzgetrf_table\b"),
    ("ssytrf_table", "dsytrf_table", "csytrf_table", r"\bzsytrf_table\b"),
    ("shetrf_table", "dhetrf_table", "chetrf_table", r"\bzhetrf_table\b"),
    ("spxtrf_table", "dpxtrf_table", "cpxtrf_table", r"\bzpxtrf_table\b"),
    ("strsm_table", "dtrsm_table", "ctrsm_table", r"\bztrsm_table\b"),
    ("sdiag_table", "ddiag_table", "cdiag_table", r"\bzdiag_table\b"),
]

# Mixed sources (zc -> ds): double-complex input, single-complex factors.
MIXED = [
    ("double", r"\bpastix_complex64_t\b"),
    ("float", r"\bpastix_complex32_t\b"),
    ("double", r"\bspm_complex64_t\b"),
    ("coeftab_dcblk", r"coeftab_zcblk"),
    ("coeftab_ds", r"coeftab_zc"),
    ("cpucblk_ds", r"cpucblk_zc"),
    ("pastix_dscores", r"pastix_zccores"),
    ("pastix_dcores", r"pastix_zcores"),
    ("pastix_dlrcores", r"pastix_zlrcores"),
    ("pastix_scores", r"pastix_ccores"),
    ("pastix_slrcores", r"pastix_clrcores"),
    ("coeftab_d", r"coeftab_z"),
    ("coeftab_s", r"coeftab_c"),
    ("cpucblk_d", r"cpucblk_z"),
    ("cpucblk_s", r"cpucblk_c"),
    ("DSOVERFCHECK", r"\bZCOVERFCHECK\b"),
    ("LAPACKE_dlag2s", r"\bLAPACKE_zlag2c"),
    ("LAPACKE_slag2d", r"\bLAPACKE_clag2z"),
    ("", r"\bconj\b"),
]


def _compiled(rules):
    return [(re.compile(r[-1]), r[:-1]) for r in rules]


NORMAL_C = _compiled(NORMAL)
MIXED_C = _compiled(MIXED)


def convert(text, prec, mixed=False):
    """Return `text` (a z or zc source) rewritten for precision `prec`."""
    if mixed:
        for rx, (ds,) in MIXED_C:
            text = rx.sub(ds, text)
        return text
    if prec == "z":
        return text
    col = PRECS.index(prec)
    for rx, repl in NORMAL_C:
        text = rx.sub(repl[col], text)
    return text


def out_name(base, prec, mixed=False):
    if mixed:
        return base.replace("zc", "ds", 1)
    # first 'z' that marks the precision in the file name
    for pat in ("_z", "z_"):
        i = base.find(pat)
        if i >= 0:
            j = i + (1 if pat == "_z" else 0)
            return base[:j] + prec + base[j + 1:]
    raise ValueError(base)


def main(argv):
    refroot, outroot = argv[1], argv[2]
    jobs = argv[3:]
    for job in jobs:
        path, precs = job.split(":")
        src = os.path.join(refroot, path)
        text = open(src).read()
        mixed = precs == "ds"
        d = os.path.join(outroot, os.path.dirname(path))
        os.makedirs(d, exist_ok=True)
        for p in (["ds"] if mixed else list(precs)):
            name = out_name(os.path.basename(path), p, mixed)
            dst = os.path.join(d, name)
            new = convert(text, p, mixed)
            if not os.path.exists(dst) or open(dst).read() != new:
                with open(dst, "w") as f:
                    f.write(new)


if __name__ == "__main__":
    main(sys.argv)
