"""Host check of the fitter's quotient sequence (Markstein's correction)
against IEEE division, with the C source in tests/native (no GPU)."""
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent


def test_markstein_quotients_are_correctly_rounded(tmp_path):
    exe = tmp_path / "markstein_check"
    cc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-fno-fast-math", str(HERE / "native" / "markstein_check.c"),
                    "-o", str(exe), "-lm"], check=True)
    r = subprocess.run([str(exe), "20000000"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip().splitlines()[-1] == "0", r.stdout
