"""Writes the compiled-model dumps the CPU reference arm of bench.py steps
(oracle/models/*.dump), so that timing the oracle never loads the product
library: the dump is the text form of mjb200_model_dump (one line per array:
name, kind i/f, count, values), produced once here from the procedural MJCF.

    python oracle/make_model_dumps.py
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "mujoco-mlx-cpp_b200"))

DUMPS = {
    "quadruped12.dump": lambda models: models.quadruped_xml(),
}


def main() -> None:
    import ctypes as C

    import mjb200

    os.makedirs(os.path.join(HERE, "models"), exist_ok=True)
    for name, make in DUMPS.items():
        m = mjb200.load_model_from_string(make(mjb200.models))
        n = mjb200.capi.lib.mjb200_model_dump(m.handle, None, 0)
        buf = C.create_string_buffer(n)
        mjb200.capi.lib.mjb200_model_dump(m.handle, buf, n)
        with open(os.path.join(HERE, "models", name), "w") as f:
            f.write(buf.value.decode())
        print("wrote", name, n, "bytes")


if __name__ == "__main__":
    main()
