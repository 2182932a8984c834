"""The enqueue trace (--qtrace) on a B200: the twins front-end's trace file equals, line for line,
the one the reference's own build writes (oracle/_ref/twins, built from the reference's sources)
on the same world: every enqueue's time, node, device, endpoints, kind, sequence number and
queue length."""
import subprocess

import pytest

from conftest import GOLDEN, ROOT, manifest
from twins_b200 import workloads

pytestmark = pytest.mark.gpu

REF = ROOT / "oracle" / "_ref" / "twins"
OURS = ROOT / "twins_b200" / "lib" / "twins"


def traces(tmp_path, args, flows, until_ps):
    out = {}
    for name, exe in (("ours", OURS), ("ref", REF)):
        q = tmp_path / f"{name}.qt"
        subprocess.run([str(exe), *args, f"--flows={flows}", f"--out={tmp_path / (name + '.csv')}", f"--qtrace={q}",
                        f"--qtrace_until={until_ps}"], check=True, capture_output=True, text=True, timeout=600)
        out[name] = q.read_text().splitlines()
    return out["ours"], out["ref"]


@pytest.mark.skipif(not REF.exists(), reason="the reference's build (make -C oracle ref) is not here")
def test_qtrace_c1_equals_reference(native_lib, tmp_path):
    flows = tmp_path / "c1.csv"
    workloads.c1()[0].flows.write_csv(flows)
    ours, ref = traces(tmp_path, ["--k=4", "--tcp=dctcp", "--ecnK=30", "--queue=200"], flows, 2_000_000_000)
    assert len(ours) > 100_000
    assert ours == ref


@pytest.mark.skipif(not REF.exists(), reason="the reference's build (make -C oracle ref) is not here")
@pytest.mark.parametrize("name", ["k8_a2a30_cubic_spray", "jf32f_a2a50_dctcp_spray"])
def test_qtrace_window_equals_reference(native_lib, tmp_path, name):
    """A window of a golden case (spraying; a topology file with link failures)."""
    case = next(c for c in manifest() if c["name"] == name)
    args = [a.replace("topo/", str(GOLDEN / "topo") + "/") for a in case["args"]] + [f"--tcp={case['tcp']}"]
    ours, ref = traces(tmp_path, args, GOLDEN / case["flows"], 300_000_000)
    assert len(ours) > 1000
    assert ours == ref
