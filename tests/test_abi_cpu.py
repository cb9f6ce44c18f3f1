"""The C-ABI library loads on any host and exports every symbol its header declares.

No compute call is made here (no GPU needed): the check is on the shared
object's dynamic symbol table against include/chameleon_b200.h, and on the
enum values the reference defines (include/chameleon/constants.h).
"""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "chameleon_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = "\n".join(l for l in txt.splitlines() if not l.lstrip().startswith(("typedef", "#")))
    names = set()
    for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", txt, flags=re.M):
        name = m.group(1)
        if name in ("if", "while", "return", "sizeof") or name.startswith("_") and not name.startswith("__chameleon"):
            continue
        names.add(name)
    # function-pointer typedefs are not functions
    return sorted(n for n in names if not n.endswith("_fct_t"))


def test_header_declares_the_reference_entry_points():
    names = set(declared_functions())
    for n in ["CHAMELEON_dposv_Tile", "CHAMELEON_dpotrf_Tile", "CHAMELEON_dpotrs_Tile", "CHAMELEON_dposv",
              "CHAMELEON_dpotrf_batch_Tile", "CHAMELEON_dtrsm_batch_Tile", "CUDA_dgemm", "CUDA_dsyrk",
              "CUDA_dtrsm", "CUDA_dpotrf", "CHAMELEON_Desc_Create", "__chameleon_init"]:
        assert n in names, n


def test_library_exports_every_declared_symbol():
    import chameleon_b200 as cb
    lib = ctypes.CDLL(cb.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert not cb.missing_symbols()


def test_enum_values_match_reference():
    import chameleon_b200 as cb
    assert (cb.ChamNoTrans, cb.ChamTrans, cb.ChamConjTrans) == (111, 112, 113)
    assert (cb.ChamUpper, cb.ChamLower, cb.ChamUpperLower) == (121, 122, 123)
    assert (cb.ChamNonUnit, cb.ChamUnit, cb.ChamLeft, cb.ChamRight) == (131, 132, 141, 142)
    assert cb.ChamRealDouble == 7 and cb.ChamRealFloat == 6


def test_compute_without_gpu_fails_loudly():
    """No CPU fallback: without a device, init reports the error instead of computing."""
    import torch
    import chameleon_b200 as cb
    if torch.cuda.is_available():
        return
    lib = cb.lib()
    assert lib.CHAMELEON_Initialized() == 0
    assert lib.__chameleon_init(1, 1) == cb.CHAMELEON_ERR_NOT_INITIALIZED
    try:
        cb.init()
    except cb.ChameleonError:
        pass
    else:
        raise AssertionError("init succeeded without a GPU")
