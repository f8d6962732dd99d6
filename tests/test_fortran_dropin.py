"""The Fortran plugin directory is a drop-in: every symbol that the reference files kept in a GPU
build import from a kernel_* or timedisc_* module (tests/golden/fortran_uses.json, extracted from
the reference by tests/golden/make_fortran_uses.py) is exported by a module of this repository's
Fortran directory or by one of the reference's own CPU time-integrator files that the build keeps,
and INTEGRATION.md's preproc.py adds exactly those files.  No Fortran compiler exists in this image,
so this is a source-level check: a module-level scan of declarations, procedures, interfaces and
types, with private/public statements honoured."""
import glob
import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FORTRAN = os.path.join(ROOT, "nemo_b200", "fortran")

# Conditions under which a use is compiled only for a kernel that this directory does not claim to
# replace: the DG/FV-smoothing kernel (PP_KERNEL_DGFV), which is absent from the reference snapshot.
NOT_THIS_KERNEL = ("PP_KERNEL_DGFV",)

# The modules a GPU build takes from the reference's own low-storage RK 4-5 directory.
KEPT = ("timedisc_const_mod", "timedisc_types_mod", "timedisc_evolve_mod", "timedisc_probe_mod")


def scan_module(path):
    """(module name, exported names) of one Fortran module file."""
    mod, names, public, default_private = None, set(), set(), False
    depth = 0          # procedure nesting
    block = None       # 'type' / 'interface' block at module level
    with open(path) as fh:
        for line in fh:
            code = line.split("!")[0].strip()
            low = code.lower()
            if not low or low.startswith("#"):
                continue
            m = re.match(r"module\s+(\w+)$", low)
            if m:
                mod = m.group(1)
                continue
            if depth == 0 and block is None:
                if low == "private":
                    default_private = True
                    continue
                m = re.match(r"public\s*::\s*(.*)$", low)
                if m:
                    public.update(x.strip() for x in m.group(1).split(","))
                    continue
                m = re.match(r"interface\s+(\w+)", low)
                if m:
                    names.add(m.group(1))
                    block = "interface"
                    continue
                if low == "interface":
                    block = "interface"
                    continue
                m = re.match(r"type\s*(?:,[^:]*)?::\s*(\w+)", low)
                if m:
                    names.add(m.group(1))
                    block = "type"
                    continue
            if block and re.match(r"end\s+" + block, low):
                block = None
                continue
            m = re.match(r"(?:pure\s+|elemental\s+|recursive\s+)*(subroutine|function)\s+(\w+)", low)
            if m:
                if depth == 0 and block is None:
                    names.add(m.group(2))
                depth += 1
                continue
            if re.match(r"end\s+(subroutine|function)", low):
                depth -= 1
                continue
            if depth == 0 and block is None and "::" in code and not low.startswith("use"):
                for part in re.split(r",(?![^(]*\))", code.split("::", 1)[1]):
                    n = re.match(r"\s*(\w+)", part)
                    if n:
                        names.add(n.group(1).lower())
    exported = {n for n in names if (n in public or not default_private)}
    return mod, exported


def our_modules():
    out = {}
    for path in glob.glob(os.path.join(FORTRAN, "**", "*.f90"), recursive=True):
        mod, exported = scan_module(path)
        assert mod, path
        out[mod] = (os.path.relpath(path, ROOT), exported)
    return out


def load_uses():
    with open(os.path.join(ROOT, "tests", "golden", "fortran_uses.json")) as f:
        return json.load(f)


def test_every_imported_kernel_and_timedisc_symbol_resolves():
    data = load_uses()
    ours = our_modules()
    kept = {m: set(v["symbols"]) for m, v in data["kept_reference_modules"].items()}
    assert set(kept) == set(KEPT)
    required = [u for u in data["uses"] if not any(c in " ".join(u["condition"]) for c in NOT_THIS_KERNEL)]
    assert len(required) >= 30
    missing = []
    for u in required:
        mod, sym = u["module"], u["symbol"].lower()
        if mod in ours:
            ok = sym in ours[mod][1]
        else:
            ok = mod in kept and sym in kept[mod]
        if not ok:
            missing.append(f"{mod}::{u['symbol']} ({u['where']})")
    assert not missing, missing
    # a module must come from one place only: ours replace the CPU kernel's, never the kept files
    assert not set(ours) & set(KEPT)


def test_symbols_the_gpu_modules_add_for_setups_and_the_mesh():
    ours = our_modules()
    share = ours["kernel_share_mod"][1]
    assert {"nodes", "weights", "refinemat", "coarsemat", "dtmin", "lmax"} <= share
    assert "dgfv_qmax" in ours["kernel_const_mod"][1]
    assert {"repair_decr", "lofactor"} <= ours["kernel_config_mod"][1]
    assert ours["kernel_validate_mod"][1] == {"kernel_repair", "kernel_validate"}
    assert {"kernel_amr_refine", "kernel_amr_coarsen"} <= ours["kernel_amr_mod"][1]
    assert {"payload_hydro_t", "auxiliary_hydro_t"} <= ours["kernel_types_mod"][1]
    assert "hook_mid_rk_timestep_500" in ours["timedisc_hooks_mod"][1]
    assert {"hook_init_400", "hook_pre_rk_timestep_300"} <= ours["kernel_hooks_mod"][1]
    assert "hook_calc_timestep_200" in ours["kernel_timestep_mod"][1]


def test_integration_preproc_adds_the_gpu_directories_and_the_kept_files():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = text[text.index("```python", text.index("## 2.")):]
    block = block[: block.index("```", 10)]
    assert "mk.add(kernel + '/*.f90')" in block and "mk.add(timedisc + '/*.f90')" in block
    assert "rk45     = home + '/source/timedisc/rungekutta/low-storage/4-5'" in block
    for m in KEPT:
        assert f"mk.add(rk45 + '/{m}.f90')" in block, m
    assert "kernel/mcfv" not in block      # no CPU kernel module is mixed in any more
