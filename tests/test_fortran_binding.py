"""The Fortran binding module (sod2d_b200/fortran/mod_sod_gpu.f90) against
the C header: every entry point of include/sod2d_gpu.h has exactly one
interface with bind(C, name=...), the same dummy arguments in the same
order, and for each argument the iso_c_binding kind and passing mode the C
type needs (scalars by value, device addresses as type(c_ptr) by value,
structs and host outputs by reference).  The image has no Fortran compiler,
so this is the check that keeps the two in step."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
KIND = {"int": "integer(c_int)", "float": "real(c_float)", "double": "real(c_double)",
        "uint64_t": "integer(c_int64_t)", "size_t": "integer(c_size_t)"}
STRUCTS = {"sod_mesh_t", "sod_phys_t", "sod_solve_opts_t", "sod_solve_stats_t", "sod_rk_cfg_t"}


def c_prototypes():
    src = re.sub(r"/\*.*?\*/", " ", (ROOT / "include" / "sod2d_gpu.h").read_text(), flags=re.S)
    out = {}
    for ret, name, args in re.findall(r"\b(int|const char \*|size_t)\s*(sod_gpu_\w+)\s*\(([^;{]*?)\)\s*;", src,
                                      flags=re.S):
        params = []
        for a in " ".join(args.split()).split(","):
            a = a.strip()
            if a in ("", "void"):
                continue
            m = re.match(r"(const\s+)?(\w+)\s*(\*{0,2})\s*(\w+)$", a)
            assert m, a
            params.append((m.group(2), m.group(3), m.group(4)))
        out[name] = (ret.strip(), params)
    return out


def f90_interfaces():
    text = (ROOT / "sod2d_b200" / "fortran" / "mod_sod_gpu.f90").read_text()
    text = re.sub(r"&\s*\n\s*", " ", text)  # join continuation lines
    out = {}
    for m in re.finditer(r"^[ \t]*([^\n!]*?)function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name='(\w+)'\)\s*\n(.*?)end function",
                         text, flags=re.S | re.M):
        ret, fname, args, cname, body = m.groups()
        if not cname.startswith("sod_gpu_"):
            continue  # helpers of the module (libc strlen)
        assert fname == cname, (fname, cname)
        decls = {}
        for line in body.splitlines():
            d = re.match(r"\s*(.+?)\s*::\s*(.+)$", line)
            if not d or d.group(1).startswith("import"):
                continue
            for n in d.group(2).split(","):
                decls[n.strip().split("(")[0].lower()] = (d.group(1), "(*)" in n)
        names = [a.strip() for a in args.split(",") if a.strip()]
        assert cname not in out, f"{cname} bound twice"
        out[cname] = (ret.strip(), names, decls)
    return out


def test_every_entry_point_is_bound():
    c, f = c_prototypes(), f90_interfaces()
    assert len(c) >= 50
    assert set(c) == set(f), (set(c) ^ set(f))


def test_argument_kinds_and_passing_match_the_header():
    c, f = c_prototypes(), f90_interfaces()
    for name, (ret, params) in c.items():
        fret, names, decls = f[name]
        want_ret = {"int": "integer(c_int)", "size_t": "integer(c_size_t)", "const char *": "type(c_ptr)"}[ret]
        assert fret == want_ret, name
        assert [n.lower() for n in names] == [p[2].lower() for p in params], name
        for ty, stars, an in params:
            attrs, is_array = decls[an.lower()]
            where = f"{name}({an})"
            if stars == "**":
                assert attrs == "type(c_ptr), intent(out)", where
            elif stars == "*" and ty in STRUCTS:
                assert attrs.startswith(f"type({ty}), intent("), where
            elif stars == "*" and ty in ("sod_gpu_ctx", "void"):
                assert attrs == "type(c_ptr), value", where
            elif ty.endswith("_fn"):  # function-pointer typedef
                assert attrs == "type(c_funptr), value", where
            elif stars == "*":
                # device address, or a host output / host array of the C type
                assert attrs == "type(c_ptr), value" or (attrs.startswith(KIND[ty] + ", intent(")
                                                          and "value" not in attrs), where
            else:
                assert attrs == f"{KIND[ty]}, value", where
            assert not is_array or stars == "*", where


def test_host_outputs_are_by_reference():
    """The host scalars and arrays the header documents as host memory are
    Fortran variables, not device addresses."""
    f = f90_interfaces()
    host = {"sod_gpu_conjgrad_pressure": ("iters", "res_rel"), "sod_gpu_conjgrad_veloc": ("iters", "res_rel"),
            "sod_gpu_incomp_veloc_stats": ("iters", "res_rel"), "sod_gpu_comp_imex_stats": ("cg_iters", "cg_res"),
            "sod_gpu_incomp_adapt_dt": ("dt",), "sod_gpu_comp_adapt_dt": ("dt",),
            "sod_gpu_incomp_analysis": ("out",), "sod_gpu_comp_analysis": ("out",),
            "sod_gpu_analysis_noalloc": ("out",), "sod_gpu_precond_set_params": ("host_params",),
            "sod_gpu_precond_get_params": ("host_params",), "sod_gpu_precond_loss_grad": ("loss", "grad_host"),
            "sod_gpu_precond_train": ("final_loss",),
            "sod_gpu_set_halo": ("ranksToComm", "commsMemPosInLoc", "commsMemSize", "nodesToComm")}
    for name, args in host.items():
        decls = f[name][2]
        for a in args:
            assert "c_ptr" not in decls[a.lower()][0], (name, a)
