"""Copies the reference's three orchestrator-planned network trees for the
4x4 grid circuit of depth 12 (src/tn/network_grid_4x4_d12{,_split,_bisect}.json,
used by network.rs:1141-1215) into this directory, after checking each
against the SHA3-256 its test pins.  The trees are test data (JSON), read
byte for byte; run this where the reference tree is mounted:

    python tests/golden/copy_network_fixtures.py /root/reference
"""
import hashlib
import os
import sys

PINS = {  # network.rs:1142, 1164-1165, 1192-1193
    "network_grid_4x4_d12.json": "3ac1c2130343db568ea5ee2c22b6f2f7291f0d39cd3c73800aad3be734ad01ed",
    "network_grid_4x4_d12_split.json": "06ca39ca74c302b35a58990558022c0ee78fa637d9043d8b19f8814b2f4aa561",
    "network_grid_4x4_d12_bisect.json": "6038f75c8c231db5e672af5b3eb22a95968a7aabd50b170029466267e364988a",
}


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for name, digest in PINS.items():
        with open(os.path.join(ref_root, "src", "tn", name), "rb") as f:
            data = f.read()
        got = hashlib.sha3_256(data).hexdigest()
        if got != digest:
            raise SystemExit(f"{name}: sha3-256 {got} is not the pinned {digest}")
        with open(os.path.join(here, name), "wb") as f:
            f.write(data)
        print(f"{name}: {len(data)} bytes, sha3-256 {got}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
