"""The drop-in CLI (`conan ic`, `conan run`) against the files the reference's
own binary wrote for the same command lines (tests/golden/<case>.npz, made by
tests/golden/make_golden.py from the unmodified reference).

FP64 (`--precision fp64`): fields to 1e-11 and trajectories to 1e-9 of the
field / box scale (cuFFT versus the reference's FFT rounding). The default FP32
run: particle positions within a small fraction of a force cell.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "conan_b200" / "bin" / "conan"
GOLD = ROOT / "tests" / "golden"
CASES = ["c1s", "c2s", "c3s", "c4s"]


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def _run(args, cwd):
    r = subprocess.run([str(EXE), *args], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def _header_dict(lines):
    return dict(str(l).split("=", 1) for l in lines)


@pytest.mark.parametrize("name", CASES)
def test_ic_and_fp64_run_reproduce_the_reference_files(gpu, tmp_path, name):
    from conan_b200.conanfile import ConanFile
    g = np.load(GOLD / f"{name}.npz")
    _run(["ic", "-i", name, *str(g["ic_args"]).split()], tmp_path)
    ic = ConanFile.read(str(tmp_path / f"{name}.density.init.conan"))
    for rec in ("density", "potential", "displacement"):
        if rec in g.files:
            assert _rel(ic.records[rec], g[rec]) < 1e-11, rec
    ref_hdr = _header_dict(g["ic_header"])
    for k, v in ref_hdr.items():
        assert ic.header.get(k) == v, (k, ic.header.get(k), v)

    _run(["run", "-i", name, *str(g["run_args"]).split(), "--precision", "fp64"], tmp_path)
    snaps = sorted(k[3:] for k in g.files if k.startswith("pos"))
    assert snaps
    L = float(ref_hdr["size"])
    for k in snaps:
        c = ConanFile.read(str(tmp_path / f"{name}.pos.{k}.conan"))
        assert np.max(np.abs(c.records["pos"] - g[f"pos{k}"])) < 1e-9 * L, k
        assert _rel(c.records["mom"], g[f"mom{k}"]) < 1e-8, k
        for hk, hv in _header_dict(g[f"hdr{k}"]).items():
            assert c.header.get(hk) == hv, (k, hk, c.header.get(hk), hv)


@pytest.mark.parametrize("name", CASES)
def test_default_fp32_run_tracks_the_reference(gpu, tmp_path, name):
    from conan_b200.conanfile import ConanFile
    g = np.load(GOLD / f"{name}.npz")
    ic_file = tmp_path / f"{name}.density.init.conan"
    _run(["ic", "-i", name, *str(g["ic_args"]).split()], tmp_path)
    assert ic_file.exists()
    _run(["run", "-i", name, *str(g["run_args"]).split()], tmp_path)
    hdr = _header_dict(g["ic_header"])
    run_args = str(g["run_args"]).split()
    f = int(run_args[run_args.index("-f") + 1]) if "-f" in run_args else 2  # the reference's default f
    cell = float(hdr["size"]) / (int(hdr["N"]) * f)
    for k in sorted(k[3:] for k in g.files if k.startswith("pos")):
        c = ConanFile.read(str(tmp_path / f"{name}.pos.{k}.conan"))
        err = np.abs(c.records["pos"] - g[f"pos{k}"]) / cell
        print(f"{name} snapshot {k}: FP32 position error rms {np.sqrt(np.mean(err ** 2)):.2e}, "
              f"max {err.max():.2e} cells")
        assert np.sqrt(np.mean(err ** 2)) < 1e-3 and err.max() < 5e-2


def test_errors_follow_the_reference(gpu, tmp_path):
    r = subprocess.run([str(EXE), "run", "-i", "missing"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode != 0 and "[error]" in (r.stdout + r.stderr)
    r = subprocess.run([str(EXE), "nosuchcommand"], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0


@pytest.mark.parametrize("name", CASES)
def test_cic_tool_reproduces_the_reference_files(gpu, tmp_path, name):
    """`conan cic` (plain and sub-sampled) on the reference's own snapshots,
    against the density files its own `cic` wrote for the same options."""
    from conan_b200.conanfile import ConanFile
    g = np.load(GOLD / f"{name}.npz")
    keys = [k for k in g.files if k.startswith("rho") and not k.startswith("rhohdr")]
    assert keys
    for k in keys:
        snap, f, s = k[3:].split("_")
        hdr = _header_dict(g[f"hdr{snap}"])
        c = ConanFile(header=hdr)
        c.update_history("ran nbody")
        c.add("pos", g[f"pos{snap}"])
        c.add("mom", g[f"mom{snap}"])
        c.write(str(tmp_path / f"{name}.pos.{snap}.conan"))
        _run(["cic", "-i", name, "-m", snap, "-f", f[1:], "-s", s[1:]], tmp_path)
        r = ConanFile.read(str(tmp_path / f"{name}.rho.{snap}.conan"))
        assert _rel(r.records["density"], g[k]) < 1e-11, k
        assert r.header == _header_dict(g[f"rhohdr{snap}_{f}_{s}"]), k


def test_ifrit_and_ascii_snapshots(gpu, tmp_path):
    """The other two snapshot formats of the reference (src/run/nbody.hh:135-166)."""
    g = np.load(GOLD / "c3s.npz")
    _run(["ic", "-i", "c3s", *str(g["ic_args"]).split()], tmp_path)
    _run(["run", "-i", "c3s", *str(g["run_args"]).split(), "--precision", "fp64", "--ascii"], tmp_path)
    rows = np.loadtxt(tmp_path / "c3s.pos.1.txt")
    assert rows.shape == (8 ** 3, 6)
    assert np.max(np.abs(rows[:, :3] - g["pos1"])) < 1e-4 * 40  # printed with 6 significant digits
    _run(["run", "-i", "c3s", *str(g["run_args"]).split(), "--precision", "fp64", "--ifrit"], tmp_path)
    raw = (tmp_path / "c3s.pos.1.bin").read_bytes()
    n = np.frombuffer(raw[4:8], dtype=np.uint32)[0]
    assert n == 8 ** 3
    off = 4 + 4 + 4 + (4 + 24 + 4)
    x = np.frombuffer(raw[off + 4: off + 4 + 4 * n], dtype=np.float32)
    assert np.allclose(x, g["pos1"][:, 0], rtol=1e-6, atol=1e-5)


def _fof_blocks(text):
    lines = text.split("\n")
    h = lines.index("# history")
    e = lines.index("", h)
    header = dict(l[2:].split("=", 1) for l in lines[1:h - 1])
    history = lines[h + 1:e]
    return header, history, "\n".join(lines[e + 1:])


@pytest.mark.parametrize("name", [str(c) for c in np.load(GOLD / "fof.npz")["cases"]])
def test_fof_tool_reproduces_the_reference_files(gpu, tmp_path, name):
    """`conan fof -f <snapshot> -i <id> -l <ll>` on the reference's snapshots
    against the text files its own `fof` wrote: the same groups and lines byte
    for byte, the same header keys (the input path aside), the same history."""
    from conan_b200.conanfile import ConanFile
    g = np.load(GOLD / "fof.npz")
    snap = str(g[f"{name}_snapshot"])
    if ":" in snap:
        f, k = snap.split(":")
        z = np.load(GOLD / f)
        pos, mom, hdr = z[k], z["mom" + k[3:]], z["hdr" + k[3:]]
    else:
        pos, mom, hdr = g[snap], g[snap.replace("_pos", "_mom")], g[snap.replace("_pos", "_hdr")]
    c = ConanFile(header=_header_dict(hdr), history=[(1700000000, "ran nbody")])
    c.add("pos", pos)
    c.add("mom", mom)
    c.write(str(tmp_path / "snap.conan"))
    _run(["fof", "-f", str(tmp_path / "snap.conan"), "-i", name, "-l", str(g[f"{name}_ll"])], tmp_path)
    got = (tmp_path / f"{name}.fof.10000.txt").read_text()
    gh, ghist, gbody = _fof_blocks(got)
    rh, rhist, rbody = _fof_blocks(str(g[f"{name}_text"]))
    assert gbody == rbody
    gh.pop("filename"), rh.pop("filename")
    assert gh == rh
    assert ghist[0] == rhist[0] and len(ghist) == len(rhist) == 2
    assert ghist[1].split(":", 1)[1].split()[0] == "fof"
