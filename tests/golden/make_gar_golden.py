"""Writes tests/golden/gar_helpers.json: outputs of the reference's own GAR
filter helpers (label hash table, bitmap popcount, 7-entry heap) on fixed
inputs, from oracle/_ref/ref_gar_helpers built by oracle/build_ref.sh against
the reference sources.  Run here, where the reference is mounted; the tests
read only the committed JSON."""
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    subprocess.run(["sh", os.path.join(ROOT, "oracle", "build_ref.sh")], check=True)
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gar_helpers")
    out = json.loads(subprocess.run([exe], capture_output=True, text=True, check=True).stdout)
    out["source"] = ("oracle/ref_gar_helpers.cu compiled against core/data_structures/heap.cuh, "
                     "core/data_structures/mini_kernel_bitmap.cuh and "
                     "core/task/gpu_task/kernel/algorithms/hash.cuh of the reference")
    with open(os.path.join(HERE, "gar_helpers.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")


if __name__ == "__main__":
    main()
