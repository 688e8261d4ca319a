"""The reference-side binding, compiled: the reference's own src/main.cpp,
src/io.cpp and src/async_output.cpp, unmodified, linked with
adaptflood_b200/binding/kernels_af.cpp in place of src/kernels.cpp and with
libadaptflood.so (oracle/_ref/lisflood_af; the Kokkos-API shim allocates the
CudaUVMSpace views in managed memory, as Kokkos' CUDA backend does).

The same .par case run by that binary (the reference's loop on this
library's CUDA kernels, its call sites src/main.cpp:231,236,267,271,281,285,
339,382 untouched) and by the reference's CPU build (oracle/_ref/lisflood_ref)
writes the same files: identical headers, values within the last printed
digit of "%.4f", the same stage.csv.
"""
import os
import subprocess

import pytest

from oracle import oracle as orc
from test_output_gpu import STAGES, _case, _compare_with_reference, _run_reference

pytestmark = pytest.mark.gpu

BINDING_CLI = os.path.join(os.path.dirname(orc.REF_CLI), "lisflood_af")


@pytest.mark.parametrize("voutput,async_out", [(True, True), (False, False)])
def test_reference_main_on_the_binding_matches_reference_cli(cuda, tmp_path, voutput,
                                                             async_out):
    if not (os.path.exists(orc.REF_CLI) and os.path.exists(BINDING_CLI)):
        pytest.skip("reference CLI or binding CLI not built")
    case = _case()
    ref_dir = _run_reference(case, str(tmp_path), voutput, async_out)
    par = os.path.join(str(tmp_path), "ref_in", "case.par")
    ours = str(tmp_path / "binding_out")
    mine = os.path.join(str(tmp_path), "binding.par")
    with open(par) as f, open(mine, "w") as g:
        for line in f:
            g.write(f"dirroot {ours}\n" if line.startswith("dirroot") else line)
    os.makedirs(ours, exist_ok=True)  # the reference opens stage.csv before it creates dirroot
    r = subprocess.run([BINDING_CLI, mine], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert len(STAGES) == 3
    _compare_with_reference(case, ref_dir, ours)
