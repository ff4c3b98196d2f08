"""The C++ drop-in shim (gtom_b200/shim/gtom_rln_shim.cu) defines gtom's own
symbols.

The shim is compiled against the reference's headers and its defined
`gtom::` symbols are compared, mangled, with those of the reference's own
objects (oracle/_ref/obj/, compiled from the reference sources by
`make -C oracle ref`): every function of include/Relion.cuh that the
reference defines in the replaced files, and d_ReconstructGridding
(include/Reconstruction.cuh:16), must be defined by the shim under the same
mangled name, so that callers link against the shim unchanged.  The two
functions the reference declares but never defines
(d_rlnSquaredDifferences, d_rlnSquaredDifferencesSparse) are defined by the
shim as well.  Every C entry point the shim calls must be exported by
libgtomrln.so.

Needs the reference tree (GTOM_REFERENCE, else the checkout the build
entry point uses) and its built objects; skipped without them.
"""
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SHIM = ROOT / "gtom_b200" / "shim" / "gtom_rln_shim.cu"
REF_OBJ = ROOT / "oracle" / "_ref" / "obj"
# reference translation units the shim replaces (oracle/_ref/obj names)
REPLACED = ["Relion_Project", "Relion_Backproject", "Relion_ProjectShifted", "Relion_BackprojectShifted",
            "Relion_BackprojectTomo", "Relion_ConvertWeights", "Relion_DiffRemap", "Relion_Misc",
            "Relion_StoreWeights"]
DECLARED_ONLY = {"d_rlnSquaredDifferences", "d_rlnSquaredDifferencesSparse"}


def reference_tree() -> Path:
    sys.path.insert(0, str(ROOT))
    import __graft_entry__
    return __graft_entry__.REFERENCE


def defined(obj: Path) -> dict[str, str]:
    """Mangled -> demangled for the gtom::d_* API functions an object defines
    (the host stubs of its __global__ kernels are left out)."""
    out = subprocess.run(["nm", "--defined-only", str(obj)], capture_output=True, text=True, check=True).stdout
    mangled = [ln.split()[-1] for ln in out.splitlines() if " T " in ln and ln.split()[-1].startswith("_ZN4gtom")]
    dem = subprocess.run(["c++filt"], input="\n".join(mangled), capture_output=True, text=True, check=True).stdout
    return {m: d for m, d in zip(mangled, dem.splitlines()) if name_of(d).startswith("d_")}


def name_of(demangled: str) -> str:
    return demangled.split("(")[0].split("::")[-1]


@pytest.fixture(scope="module")
def shim_obj(tmp_path_factory):
    ref = reference_tree()
    if not (ref / "include" / "Relion.cuh").exists():
        pytest.skip("reference headers not present")
    obj = tmp_path_factory.mktemp("shim") / "gtom_rln_shim.o"
    subprocess.run(["nvcc", "-std=c++14", "-w", "-c", str(SHIM), "-o", str(obj), "-I", str(ref / "include"),
                    "-I", str(ROOT / "include"), "-Xcompiler", "-fPIC"], check=True, capture_output=True)
    return obj


def test_shim_defines_the_reference_symbols(shim_obj):
    if not all((REF_OBJ / f"{n}.o").exists() for n in REPLACED + ["Reconstruction_RecFourier"]):
        pytest.skip("reference objects not built (make -C oracle ref)")
    want = {}
    for n in REPLACED:
        want.update(defined(REF_OBJ / f"{n}.o"))
    grid = {m: d for m, d in defined(REF_OBJ / "Reconstruction_RecFourier.o").items()
            if name_of(d) == "d_ReconstructGridding"}
    assert len(grid) == 1
    want.update(grid)
    got = defined(shim_obj)
    missing = sorted(d for m, d in want.items() if m not in got)
    assert not missing, f"shim lacks: {missing}"
    extra = sorted(d for m, d in got.items() if m not in want and name_of(d) not in DECLARED_ONLY)
    assert not extra, f"shim defines symbols the reference does not: {extra}"
    assert {name_of(d) for m, d in got.items() if m not in want} == DECLARED_ONLY
    assert len(want) == 23  # 4 + 2 + 2 + 2 + 4 + 4 + 2 + 1 + 1 overloads, and the gridding


def test_shim_calls_only_exported_entry_points(shim_obj, gtom_lib):
    from gtom_b200 import _lib
    und = subprocess.run(["nm", "--undefined-only", str(shim_obj)], capture_output=True, text=True,
                         check=True).stdout
    called = {ln.split()[-1] for ln in und.splitlines() if ln.split()[-1].startswith("gtomrln_")}
    assert len(called) >= 25
    exported = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                              check=True).stdout
    names = {ln.split()[-1] for ln in exported.splitlines()}
    assert called <= names, sorted(called - names)
