"""The C-ABI library loads and exports every symbol its headers declare
(no compute call: this runs without a GPU)."""
import ctypes
import os
import subprocess

import pytest

import ggms_b200


def test_library_built():
    assert os.path.exists(ggms_b200.LIB_PATH), "run make -C ggms-distributed_b200"


def test_every_declared_symbol_exported():
    lib = ggms_b200.load()
    names = ggms_b200.declared_symbols()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_no_undeclared_exports():
    out = subprocess.run(["nm", "-D", "--defined-only", ggms_b200.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l and "ggms_" in l}
    assert exported <= set(ggms_b200.declared_symbols()), exported - set(ggms_b200.declared_symbols())


def test_status_strings_and_version():
    lib = ggms_b200.load()
    assert lib.ggms_version() >= 100
    assert ggms_b200.status_string(0) == "ok"
    assert ggms_b200.status_string(1) == "invalid argument"


def test_default_opts_layout():
    o = ggms_b200.default_opts()
    assert o.struct_size == ctypes.sizeof(ggms_b200.Opts)
    assert o.assigner == ggms_b200.ASSIGNER_AUTO
    assert o.pl_knots == 0


def test_struct_layouts_match_the_header(tmp_path):
    """The binding's ctypes structs have the C header's sizes and offsets
    (compiled here with gcc against include/ggms.h)."""
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "ggms.h"\n'
        'int main(void) { printf("%zu %zu %zu %zu %zu\\n", sizeof(ggms_opts), offsetof(ggms_opts, stats),'
        ' offsetof(ggms_opts, pl_knots), sizeof(ggms_stats), offsetof(ggms_stats, window_runs));'
        ' return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    O, S = ggms_b200.Opts, ggms_b200.Stats
    assert got == [ctypes.sizeof(O), O.stats.offset, O.pl_knots.offset, ctypes.sizeof(S),
                   S.window_runs.offset]




def test_generate_rejects_before_launch():
    """Argument checks of the device generators return before any CUDA call."""
    lib = ggms_b200.load()
    fake = ctypes.c_void_p(0x1000)            # never dereferenced: every case returns early
    for suf, kinds in (("f32", 10), ("f64", 3), ("u32", 3)):
        fn = getattr(lib, f"ggms_generate_{suf}")
        assert fn(None, 16, 0, 1, None) == 1
        assert fn(fake, 0, 0, 1, None) == 1
        assert fn(fake, 16, -1, 1, None) == 1
        assert fn(fake, 16, kinds, 1, None) == 1
    assert lib.ggms_generate_f32(fake, 1 << 31, 2, 1, None) == 5    # KILLER FLOATS: CUB's int count
    assert lib.ggms_generate_f64(fake, 1 << 31, 2, 1, None) == 5    # KILLER DOUBLES
    assert lib.ggms_generate_f32(fake, (1 << 32) + 1, 8, 1, None) == 5
    assert lib.ggms_generate_u32(fake, (1 << 32) + 1, 1, 1, None) == 5


def test_package_never_reaches_the_oracle():
    """The product (the CUDA library and its Python binding) has no path to the CPU
    oracle: no import of it, no load of its library, no link against it."""
    pkg = os.path.dirname(ggms_b200.__file__)
    csrc = os.path.join(os.path.dirname(pkg), "csrc")
    files = [os.path.join(pkg, f) for f in os.listdir(pkg) if f.endswith(".py")]
    files += [os.path.join(csrc, f) for f in os.listdir(csrc)]
    files.append(os.path.join(os.path.dirname(pkg), "Makefile"))
    for path in files:
        with open(path) as f:
            txt = f.read()
        for needle in ("ggms_oracle", "libggms_ref", "oracle/"):
            assert needle not in txt, (path, needle)
