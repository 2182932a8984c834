"""The reference's two parameter sweeps as batches of worlds on a B200, against sequential ns-3.

The reference checks its batching path this way (validation/check_sweeps.sh with bench/sweep.py):
every ecnK x queue x TCP configuration of FatTree k=8 (138, flows k8_a2a30 and k8_a2a50w) and of
k=16 (48, flows k16_a2a30 and k16_a2a50w) runs as a world of a batch, and each world's
established and completed times must equal the stored ns-3 output. Worlds whose ties the 9-run
chains could not decide run again on the 25-run build, as bench/sweep.py reruns them on twins128.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN
from twins_b200 import api

pytestmark = pytest.mark.gpu

INDEX = json.loads((GOLDEN / "sweep" / "index.json").read_text())


def expected(sweep):
    z = np.load(GOLDEN / "sweep" / f"{sweep}.npz")
    est, done, out, at = z["est"], z["done"], [], 0
    for c in INDEX[sweep]:
        out.append((est[at:at + c["rows"]], done[at:at + c["rows"]]))
        at += c["rows"]
    return out


def world(c):
    topo = api.Topology.fattree(c["k"])
    flows = api.Flows.load(GOLDEN / c["flows"], topo.hosts)
    return topo, flows, api.TcpParams(c["tcp"], c["ecn_k"], c["queue"])


def run_batch(configs, chain_runs=9):
    with api.Simulator(chain_runs=chain_runs) as sim:
        ids = [sim.add_world(*world(c)) for c in configs]
        sim.run()
        return [sim.results(i) for i in ids], [sim.counters(i)["undecided_ties"] for i in ids], sim.stats()


@pytest.mark.parametrize("sweep,batch", [("k8", 138), ("k16", 48)])
def test_sweep_batch_equals_ns3(native_lib, sweep, batch):
    configs, want = INDEX[sweep], expected(sweep)
    same, redo = 0, []
    for b in range(0, len(configs), batch):
        part = configs[b:b + batch]
        res, ties, _ = run_batch(part)
        for j, c in enumerate(part):
            if ties[j]:
                redo.append(b + j)
                continue
            ok = (res[j][0] == want[b + j][0]).all() and (res[j][1] == want[b + j][1]).all()
            assert ok, f"{c['name']}: {int(((res[j][0] != want[b + j][0]) | (res[j][1] != want[b + j][1])).sum())} flows differ"
            same += 1
    if redo:
        res, ties, _ = run_batch([configs[i] for i in redo], chain_runs=25)
        for j, i in enumerate(redo):
            assert ties[j] == 0, f"{configs[i]['name']}: ties undecided with 25-run chains too"
            assert (res[j][0] == want[i][0]).all() and (res[j][1] == want[i][1]).all(), configs[i]["name"]
            same += 1
    assert same == len(configs)
