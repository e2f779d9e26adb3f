"""The C ABI on the CPU: the library loads, exports exactly what
include/beagle_b200.h declares, and refuses cleanly without a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "beagle_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(beagleB200\w+)\s*\(", text)))


def test_header_declares_the_hot_path():
    names = declared()
    for need in ["beagleB200CreateInstance", "beagleB200UpdateTransitionMatrices",
                 "beagleB200UpdatePartials", "beagleB200UpdatePrePartials",
                 "beagleB200AccumulateScaleFactors", "beagleB200CalculateRootLogLikelihoods",
                 "beagleB200CalculateEdgeDerivatives", "beagleB200SetTipStates"]:
        assert need in names


def test_library_exports_every_declared_symbol(pkg):
    if not os.path.exists(pkg.LIB_PATH):
        pytest.fail("libbeagle_b200.so not built")
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (beagleB200\w+)", out))
    assert set(declared()) == exported
    lib = ctypes.CDLL(pkg.LIB_PATH)
    for name in declared():
        assert getattr(lib, name) is not None


def test_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "beagle_b200.h"\nint main(void){return BEAGLE_B200_OP_COUNT-7;}\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                    str(src), "-o", str(tmp_path / "t")], check=True)


def test_binding_table_covers_header(pkg):
    bound = set("beagleB200" + n for n in pkg.binding._SIGS)
    bound |= set("beagleB200" + n for n in pkg.binding._BATCH_SIGS)
    bound |= {"beagleB200CreateInstance", "beagleB200GetResourceList", "beagleB200GetVersion"}
    # bound directly by its own test (raw device pointers, no instance)
    bound |= {"beagleB200RootLogLikelihoodsNoAlloc"}
    assert set(declared()) <= bound


def test_no_gpu_is_a_clean_error(pkg):
    """Without a CUDA device the library reports NO_RESOURCE instead of
    falling back to anything."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = pkg.load()
    assert lib.resources() == []
    with pytest.raises(pkg.binding.BeagleError) as e:
        lib.create(4, 7, 4, 4, 10, 1, 6, 1, 0)
    assert e.value.code == -6
