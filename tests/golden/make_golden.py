"""Copies the reference's regression histories for the compressible and
incompressible Taylor-Green tests into this folder as fixtures.

Each file holds rows of (time, EK, eps_S, eps_D, eps_T, max Mach) written by
the reference's write_EK (src/lib_sod2d/sources/mod_analysis.f90:170-185),
one row at t=0 and one every 10 steps.  Source paths are relative to the
reference project.  Run with the reference checked out at the given root:

    python tests/golden/make_golden.py /path/to/sod2d
"""
import shutil
import sys
from pathlib import Path

SOURCES = {
    "tgv_comp_cpu_lsrk5_8x8x8_p4.dat": "Tests/TGV_Compressible/CPU/LS_RK_5/Reference/analysis_cube-4.dat",
    "tgv_comp_gpu_lsrk5_12x12x12_p4.dat": "Tests/TGV_Compressible/GPU/LS_RK_5/Reference/analysis_cube-1.dat",
    "tgv_comp_cpu_imex4_8x8x8_p4.dat": "Tests/TGV_Compressible/CPU/IMEX/Reference/analysis_cube-4.dat",
    "tgv_incomp_cpu_ab_8x8x8_p4.dat": "Tests/TGV_Incomp/CPU/AB/Reference/analysis_cube-4.dat",
    "tgv_incomp_gpu_ab_12x12x12_p4.dat": "Tests/TGV_Incomp/GPU/AB/Reference/analysis_cube-1.dat",
}

if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <root of the reference checkout>")
    root = Path(sys.argv[1])
    here = Path(__file__).resolve().parent
    for dst, src in SOURCES.items():
        shutil.copyfile(root / src, here / dst)
        print(dst, "<-", src)
