"""Golden fixtures recorded from the reference's own Host path
(tests/golden/make_golden.py): the oracle's C restatement (CPU) and the CUDA
grid (GPU) replay each scenario from its seed and must reproduce every digest
-- the inputs drawn and every array of every subdomain after every call."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import scenarios  # noqa: E402

NAMES = sorted(scenarios.SCENARIOS)


def fixture(name):
    with open(os.path.join(HERE, "golden", f"{name}.json")) as f:
        return json.load(f)


def check(fx, record, out):
    assert record == fx["inputs"], "the seeded inputs differ from the recorded ones"
    bad = sorted(k for k in fx["outputs"] if out.get(k) != fx["outputs"][k])
    assert not bad, f"{len(bad)} digests differ, first: {bad[:8]}"
    assert set(out) == set(fx["outputs"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_port_reproduces_reference_fixture(name):
    spec = scenarios.SCENARIOS[name]
    fx = fixture(name)
    grid = scenarios.make_oracle("port", spec)
    record = {}
    out = scenarios.run(grid, spec, record=record, seed=fx["seed"])
    grid.close()
    check(fx, record, out)


class GpuGrid:
    """The CUDA grid with the two helpers the scenario runner needs."""

    def __init__(self, spec):
        import dsdecompx_b200 as dsx
        self.spec = spec
        self.port = scenarios.make_oracle("port", spec)   # initial owners only
        self.g = dsx.VirtualGrid(spec["P"], spec["dims"], spec["policy"], spec["lower"],
                                 spec["upper"], spec["periodic"], spec["halo"], spec["edges"],
                                 spec["dynamic"], spec["fields"], particles=spec["N"])

    def owner_rank(self, pos):
        return self.port.owner_rank(pos)

    def __getattr__(self, name):
        return getattr(self.g, name)

    def close(self):
        self.g.close()
        self.port.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_grid_reproduces_reference_fixture(cuda, name):
    spec = scenarios.SCENARIOS[name]
    fx = fixture(name)
    grid = GpuGrid(spec)
    record = {}
    out = scenarios.run(grid, spec, record=record, seed=fx["seed"])
    grid.close()
    check(fx, record, out)
