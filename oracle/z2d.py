#!/usr/bin/env python3
"""Complex-double -> real-double source generator for the reference oracle build.

Test infrastructure only: this script turns the reference's `z`-precision C
sources (Chameleon ships only `z` files and generates `s/d/c` at build time with
an external tool whose submodule is empty in the reference tree) into
`d`-precision sources under ``oracle/_ref/gen``.  The generated files are the
reference's own code with names substituted; they are compiled by
``oracle/build_ref.sh`` into the reference CPU library that the parity tests and
the CPU baseline use.  Nothing in the product links them.

Rules written for this oracle (the reference's own rule tables live in
``cmake_modules/local_subs.py`` and the absent precision generator):

* types:   CHAMELEON_Complex64_t -> double, CHAMELEON_Complex32_t -> float,
           ChamComplexDouble -> ChamRealDouble, ChamComplexFloat -> ChamRealFloat
* macros:  CBLAS_SADDR(x) -> (x), creal(x)/conj(x) -> (x), cimag(x) -> 0
* routines: Hermitian names become symmetric names (zherk -> dsyrk, zlanhe ->
           dlansy, zplghe -> dplgsy, zhemm -> dsymm, zher2k -> dsyr2k,
           zhessq -> dsyssq), ChamHermitian -> ChamSymmetric (outside coreblas)
* every remaining identifier piece carrying the `z` precision letter in a known
  prefix (CORE_z, TCORE_z, INSERT_TASK_z, CHAMELEON_z, chameleon_pz,
  cblas_z, LAPACKE_z, codelet_z, ...) gets `d`.
* ``PRECISION_z`` / ``PRECISION_c`` guards are left intact: generated files are
  compiled with ``-DPRECISION_d`` (the reference compiles its generated files
  the same way; ``NBELEM`` in core_zplgsy.c depends on it).
"""
import os
import re
import sys

HERM = [
    ("zherk", "dsyrk"), ("ZHERK", "DSYRK"),
    ("zher2k", "dsyr2k"), ("ZHER2K", "DSYR2K"),
    ("zhemm", "dsymm"), ("ZHEMM", "DSYMM"),
    ("zlanhe", "dlansy"), ("ZLANHE", "DLANSY"),
    ("zplghe", "dplgsy"), ("ZPLGHE", "DPLGSY"),
    ("zhessq", "dsyssq"), ("ZHESSQ", "DSYSSQ"),
    ("zhe2ge", "dhe2ge"),
]

# prefixes after which a `z` / `Z` precision letter is replaced by `d` / `D`
PREFIXES = [
    "TCORE_", "CORE_", "INSERT_TASK_", "CHAMELEON_", "chameleon_p", "chameleon_",
    "cblas_", "LAPACKE_", "codelet_", "cl_", "core_", "runtime_", "RUNTIME_",
    "CUDA_", "TCUDA_", "flops_", "FLOPS_", "testing_", "check_", "workspace_",
    "coreblas_", "compute_", "tasks_", "gpucublas_", "TCUDA_", "HIP_",
    "chameleon_getaddr_", "vendor_", "morse_", "cham_", "starpu_",
]

TYPE_SUBS = [
    (r"\bCHAMELEON_Complex64_t\b", "double"),
    (r"\bCHAMELEON_Complex32_t\b", "float"),
    (r"\bChamComplexDouble\b", "ChamRealDouble"),
    (r"\bChamComplexFloat\b", "ChamRealFloat"),
    (r"\bcomplex64\b", "double"),
    (r"\bComplex64\b", "Double"),
]


def _paren_arg_sub(text, name, repl):
    """Replace NAME(arg) by repl(arg) for balanced parentheses."""
    out = []
    i = 0
    pat = re.compile(r"\b" + re.escape(name) + r"\s*\(")
    while True:
        m = pat.search(text, i)
        if not m:
            out.append(text[i:])
            break
        out.append(text[i:m.start()])
        depth = 1
        j = m.end()
        while j < len(text) and depth:
            if text[j] == "(":
                depth += 1
            elif text[j] == ")":
                depth -= 1
            j += 1
        arg = text[m.end():j - 1]
        out.append(repl(arg))
        i = j
    return "".join(out)


def convert(text, coreblas=False):
    for pat, rep in TYPE_SUBS:
        text = re.sub(pat, rep, text)
    text = _paren_arg_sub(text, "CBLAS_SADDR", lambda a: "(" + a + ")")
    text = _paren_arg_sub(text, "creal", lambda a: "(" + a + ")")
    text = _paren_arg_sub(text, "conj", lambda a: "(" + a + ")")
    text = _paren_arg_sub(text, "cimag", lambda a: "(0.0*(" + a + "))")
    for a, b in HERM:
        text = text.replace(a, b)
    if not coreblas:
        text = re.sub(r"\bChamHermitian\b", "ChamSymmetric", text)
    # prefix-driven precision letter
    for p in sorted(set(PREFIXES), key=len, reverse=True):
        text = re.sub(r"\b(" + re.escape(p) + r")z", r"\1d", text)
        text = re.sub(r"\b(" + re.escape(p) + r")Z", r"\1D", text)
    # header names: foo_z.h, foo_ztile.h
    text = re.sub(r"(\w+)_z(tile)?\.h", lambda m: m.group(1) + "_d" + (m.group(2) or "") + ".h", text)
    # remaining z-routine tokens used as plain identifiers (e.g. zone/mzone stay)
    text = re.sub(r"\bpz([a-z0-9]+)\b", r"pd\1", text)
    return text


def main():
    src_root, out_root = sys.argv[1], sys.argv[2]
    files = sys.argv[3:]
    for rel in files:
        path = os.path.join(src_root, rel)
        with open(path) as f:
            text = f.read()
        d_rel = os.path.join(os.path.dirname(rel), re.sub(r"^(\w*?)z", r"\1d", os.path.basename(rel), count=1))
        out = os.path.join(out_root, d_rel)
        os.makedirs(os.path.dirname(out), exist_ok=True)
        with open(out, "w") as f:
            f.write(convert(text, coreblas=rel.startswith("coreblas")))
        print(out)


if __name__ == "__main__":
    main()
