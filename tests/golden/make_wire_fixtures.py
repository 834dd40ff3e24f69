"""Write the CLI wire-format fixtures of tests/golden/wire/ with the reference's
own harness code (run in this container, where the reference tree exists):

* qubo_n200.bin -- the n = 200 QUBO (each pair kept with probability 0.05,
  seed 0), written by ``write_instance`` of qubo/harness/backends/praq_cuda.py;
* jrp_6x20.bin -- a 6-item, 20-period demand-driven JRP (seed 7), written by
  ``write_instance`` of jrp/harness/backends/pria_cuda.py.

The GPU tests run the file CLIs on these files, so the bytes the reference's
harness sends are the bytes the CLIs are tested on.  Usage:

    python tests/golden/make_wire_fixtures.py [/path/to/reference]
"""

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
OUT = HERE / "wire"

SNIPPET = """
import sys
sys.path.insert(0, {repo!r})
from pathlib import Path
from reformulation_b200.instances import {gen}
from harness.backends.{backend} import write_instance
write_instance({call}, Path({out!r}))
"""


def write(reference: Path, project: str, backend: str, gen: str, call: str, name: str) -> None:
    code = SNIPPET.format(repo=str(REPO), gen=gen, backend=backend, call=call, out=str(OUT / name))
    subprocess.run([sys.executable, "-c", code], check=True, cwd="/tmp",
                   env={"PYTHONPATH": str(reference / project), "PATH": "/usr/bin:/bin"})
    print(OUT / name, (OUT / name).stat().st_size, "bytes")


def main() -> None:
    reference = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    OUT.mkdir(exist_ok=True)
    write(reference, "qubo", "praq_cuda", "qubo_sparse_bernoulli", "qubo_sparse_bernoulli(0, 200, 0.05)",
          "qubo_n200.bin")
    write(reference, "jrp", "pria_cuda", "jrp_demand", "jrp_demand(7, 6, 20)", "jrp_6x20.bin")


if __name__ == "__main__":
    main()
