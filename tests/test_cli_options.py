"""The drop-in CLI keeps the reference's option tables: every option that the
reference binary's `--help` lists for `ic`, `run`, `cic` and `fof` is listed
by `conan_b200/bin/conan` with the same short name and default (options that
only this build has are extra lines). Needs no GPU: `--help` returns before
any device work."""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
OURS = ROOT / "conan_b200" / "bin" / "conan"
REF = ROOT / "oracle" / "_ref" / "conan_ref"
LINE = re.compile(r"^\s+--(\S+)(?: \| -(\S+))? \((?:default: ([^)]*)|flag)\)")
# defaults computed from the clock when the program starts (date, time-based seed)
CLOCK_DEFAULTS = {"id", "seed"}


def _options(exe, cmd):
    r = subprocess.run([str(exe), cmd, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    out = {}
    for line in r.stdout.splitlines():
        m = LINE.match(line)
        if m:
            out[m.group(1)] = (m.group(2), None if m.group(1) in CLOCK_DEFAULTS else m.group(3))
    return out


@pytest.mark.skipif(not REF.exists(), reason="reference binary not built here")
@pytest.mark.parametrize("cmd", ["ic", "run", "cic", "fof"])
def test_option_tables_match_the_reference(cmd):
    ref, ours = _options(REF, cmd), _options(OURS, cmd)
    assert len(ref) >= 5, "too few options parsed from the reference's help"
    for name, spec in ref.items():
        assert name in ours, f"{cmd}: option --{name} missing"
        assert ours[name] == spec, f"{cmd} --{name}: {ours[name]} against the reference's {spec}"
