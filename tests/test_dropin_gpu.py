"""The C++ drop-in (include/qas_mhd2d_dropin.hpp, the GpuMHD2D subclass INTEGRATION.md shows)
compiled against the reference's own 2D Orszag-Tang problem directory (2D/SERIAL/OTvortex:
mhd2d_class.hpp, its paras/init_/dout_, built at 64^2 by `make -C oracle dropin`) and linked
with libqas: its dat/ output files (params, offsets, x, y, t.dat and every outdat_*.dat state)
must be byte-identical to those of the reference's unchanged program, whose main calls
MHD2D::exec_ (mhd2d_class.cpp:35-61) where the drop-in calls exec_gpu."""
import filecmp
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
HEADER = os.path.join(ROOT, "include", "qas_mhd2d_dropin.hpp")


def test_integration_doc_shows_the_compiled_header():
    """The snippet in INTEGRATION.md is the header the check below compiles, verbatim."""
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", doc, flags=re.S)
    assert open(HEADER).read() in blocks


def _run(exe, where):
    os.makedirs(os.path.join(where, "dat"))
    r = subprocess.run([exe], cwd=where, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return sorted(os.listdir(os.path.join(where, "dat")))


@pytest.mark.gpu
def test_dropin_outputs_identical_to_reference(tmp_path):
    ref, gpu = os.path.join(REF, "dropin_ref"), os.path.join(REF, "dropin_gpu")
    if not (os.access(ref, os.X_OK) and os.access(gpu, os.X_OK)):
        pytest.skip("drop-in binaries not built (make -C oracle dropin)")
    a = _run(ref, str(tmp_path / "ref"))
    b = _run(gpu, str(tmp_path / "gpu"))
    assert a == b and len([f for f in a if f.startswith("outdat_")]) >= 3, (a, b)
    for f in a:
        assert filecmp.cmp(str(tmp_path / "ref" / "dat" / f), str(tmp_path / "gpu" / "dat" / f), shallow=False), f
