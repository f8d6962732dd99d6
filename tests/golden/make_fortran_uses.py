"""Writes fortran_uses.json: every `use kernel_*_mod, only: ...` / `use timedisc_*_mod, only: ...`
of the reference files that stay in a build with the GPU kernel directory, and the public symbols
of the reference's CPU time-integrator files that such a build keeps.

Run it where the reference tree is present (its path is the first argument); the JSON is committed
so the drop-in test (tests/test_fortran_dropin.py) runs without the reference.

Files scanned (the Euler and GLM-MHD 3D setups, the mesh layer, the driver, the FLASH checkpoint
writer, and the low-storage RK 4-5 directory whose hooks the GPU directory replaces).  Each use
records its preprocessor condition (the enclosing #if / #ifdef lines), so that uses compiled only
for kernels this build does not claim to be (PP_KERNEL_DGFV) can be told apart.

    python tests/golden/make_fortran_uses.py /root/reference
"""
import glob
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

SCAN = ["source/setups/euler/3d/**/*.f90", "source/setups/mhd/3d/**/*.f90", "source/mesh/p4est/*.f90",
        "source/driver_mod.f90", "source/checkpoint/flash/*.f90",
        "source/timedisc/rungekutta/low-storage/4-5/*.f90"]
# reference files a build with the GPU directory keeps (the 4-5 directory without its hooks)
KEPT = ["source/timedisc/rungekutta/low-storage/4-5/timedisc_const_mod.f90",
        "source/timedisc/rungekutta/low-storage/4-5/timedisc_types_mod.f90",
        "source/timedisc/rungekutta/low-storage/4-5/timedisc_evolve_mod.f90",
        "source/timedisc/rungekutta/low-storage/4-5/timedisc_probe_mod.f90"]
REPLACED = ["source/timedisc/rungekutta/low-storage/4-5/timedisc_hooks_mod.f90"]

USE = re.compile(r"^\s*use\s+((?:kernel|timedisc)_\w+_mod)\s*,\s*only\s*:\s*(.*)$", re.I)
# C preprocessor and fypp (#:if) conditionals
IF = re.compile(r"^\s*#\s*:?\s*(if|ifdef|ifndef)\b(.*)$")
ELSE = re.compile(r"^\s*#\s*:?\s*(else|elif)\b(.*)$")
ENDIF = re.compile(r"^\s*#\s*:?\s*endif\b")


def uses(root):
    out = []
    files = sorted({f for pat in SCAN for f in glob.glob(os.path.join(root, pat), recursive=True)})
    for path in files:
        rel = os.path.relpath(path, root)
        if rel in REPLACED:
            continue
        stack = []
        with open(path, errors="replace") as fh:
            for ln, line in enumerate(fh, 1):
                if IF.match(line):
                    stack.append(line.strip())
                    continue
                m = ELSE.match(line)
                if m and stack:
                    stack[-1] = stack[-1] + " / " + line.strip()
                    continue
                if ENDIF.match(line):
                    if stack:
                        stack.pop()
                    continue
                m = USE.match(line.split("!")[0])
                if not m:
                    continue
                for sym in m.group(2).split(","):
                    sym = sym.strip()
                    if "=>" in sym:
                        sym = sym.split("=>")[1].strip()
                    if sym:
                        out.append({"module": m.group(1).lower(), "symbol": sym, "where": f"{rel}:{ln}",
                                    "condition": list(stack)})
    return out


def public_symbols(path):
    """Module name and the names a module file declares at module level (variables, parameters,
    procedures, interfaces, types) -- a plain scan, enough for these small files."""
    mod, names = None, set()
    depth = 0
    with open(path, errors="replace") as fh:
        for line in fh:
            code = line.split("!")[0].strip()
            low = code.lower()
            m = re.match(r"module\s+(\w+)$", low)
            if m:
                mod = m.group(1)
                continue
            m = re.match(r"(?:pure\s+|elemental\s+|recursive\s+)*(subroutine|function)\s+(\w+)", low)
            if m:
                names.add(m.group(2))
                depth += 1
                continue
            if re.match(r"end\s+(subroutine|function)", low):
                depth -= 1
                continue
            if depth == 0 and "::" in code:
                for part in re.split(r",(?![^(]*\))", code.split("::", 1)[1]):
                    n = re.match(r"\s*(\w+)", part)
                    if n:
                        names.add(n.group(1).lower())
    return mod, sorted(names)


def main(root):
    data = {"uses": uses(root), "kept_reference_modules": {}}
    for rel in KEPT:
        mod, names = public_symbols(os.path.join(root, rel))
        data["kept_reference_modules"][mod] = {"file": rel, "symbols": names}
    with open(os.path.join(HERE, "fortran_uses.json"), "w") as f:
        json.dump(data, f, indent=1)
    print(len(data["uses"]), "uses,", len(data["kept_reference_modules"]), "kept reference modules")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
