"""Records the golden digests from the reference's own Host path.

    python tests/golden/make_golden.py

needs oracle/_ref/libdsx_ref_debug.so (built by __graft_entry__.build() from
the reference sources); writes tests/golden/<scenario>.json with the seed,
the digests of the inputs the seed draws and of every output.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import scenarios  # noqa: E402


def seed_of(name: str) -> int:
    return sum((i + 1) * ord(c) for i, c in enumerate(name))


def main():
    for name, spec in scenarios.SCENARIOS.items():
        grid = scenarios.make_oracle("ref_debug", spec)
        record = {}
        seed = seed_of(name)
        out = scenarios.run(grid, spec, record=record, seed=seed)
        grid.close()
        path = os.path.join(HERE, f"{name}.json")
        with open(path, "w") as f:
            json.dump({"scenario": name, "seed": seed, "generator": "reference Host path (oracle/_ref)",
                       "inputs": record, "outputs": out}, f, indent=0, sort_keys=True)
        print(name, os.path.getsize(path), "bytes", len(out), "output digests")


if __name__ == "__main__":
    main()
