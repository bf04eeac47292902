"""The C sample caller (astaroth_b200/csrc/ac_devicetest.c, in the shape of the
reference's samples/devicetest/main.cc): it compiles as plain C11 against the
header and links against the library on any machine; on a GPU it runs its
checks (periodic fill bit-exact, substep loop = graph step, reductions,
argument checks) and exits 0."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "astaroth_b200" / "csrc" / "ac_devicetest.c"
LIBDIR = ROOT / "astaroth_b200"


def _compile(out: Path) -> Path:
    exe = out / "ac_devicetest"
    subprocess.run(["gcc", "-O2", "-std=c11", "-Wall", "-Wextra", "-Werror",
                    f"-I{ROOT / 'include'}", str(SRC), "-o", str(exe), f"-L{LIBDIR}",
                    "-lastaroth_b200", f"-Wl,-rpath,{LIBDIR}", "-lm"], check=True)
    return exe


def test_c_sample_compiles_and_links(tmp_path):
    assert _compile(tmp_path).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [[], ["33", "24", "17"]])
def test_c_sample_runs(tmp_path, dims):
    exe = _compile(tmp_path)
    r = subprocess.run([str(exe), *dims], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "ac_devicetest: OK" in r.stdout
