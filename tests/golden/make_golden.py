"""Generates the golden fixtures in this directory from the UNMODIFIED reference.

Runs the reference's own `conan` binary (oracle/_ref/conan_ref, compiled from
the reference sources by oracle/Makefile) through its public CLI (ic, run,
cic, fof), and the
reference's own md_cic / LinearInterpolation<Gradient> templates through
oracle/_ref/libconan_ref.so, on small seeded cases. Needs the reference tree
(only in the build container); the fixtures it writes are committed.

    python tests/golden/make_golden.py          # everything
    python tests/golden/make_golden.py fof      # fof.npz only, from the committed snapshots
"""
import ctypes
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
from conan_b200.conanfile import ConanFile  # noqa: E402

REF = ROOT / "oracle" / "_ref"

# name: (ic args, run args)
CASES = {
    "c1s": ("-d 2 -b 6 -L 50 --scale-free -n -1 --potential -z --seed 1",
            "-f 1 -a0 0.02 -da 0.049 -n 20"),
    "c2s": ("-d 3 -b 4 -L 12.5 --scale-free -n -2 --smooth --scale 0.78125 --potential --seed 2",
            "-f 1 -a0 0.02 -da 0.0196 -n 20"),
    "c3s": ("-d 3 -b 3 -L 40 --scale-free -n -1.5 --potential -z --seed 3",
            "-a0 0.05 -da 0.0475 -n 10"),
    "c4s": ("-d 2 -b 5 -L 30 --potential --seed 4 --Omega0 0.3 --H0 70 -n 0.96",
            "-f 2 -c -a0 0.1 -da 0.05 -n 10"),
}

# (f, sub-sample) of the `cic` runs on every snapshot
CIC_CASES = [(2, 1), (1, 2), (2, 2)]


def run_cli(name, ic_args, run_args, work):
    exe = str(REF / "conan_ref")
    subprocess.run([exe, "ic", "-i", name, *ic_args.split()], cwd=work, check=True, stdout=subprocess.DEVNULL)
    subprocess.run([exe, "run", "-i", name, *run_args.split()], cwd=work, check=True, stdout=subprocess.DEVNULL)
    out = {}
    ic = ConanFile.read(str(Path(work) / f"{name}.density.init.conan"))
    for k, v in ic.records.items():
        out[k] = v
    out["ic_header"] = np.array(sorted(f"{k}={v}" for k, v in ic.header.items() if k != "seed" or True))
    snaps = sorted(Path(work).glob(f"{name}.pos.*.conan"))
    for s in snaps:
        k = s.name.split(".")[2]
        c = ConanFile.read(str(s))
        out[f"pos{k}"] = c.records["pos"]
        out[f"mom{k}"] = c.records["mom"]
        out[f"apos{k}"] = np.float64(c.header["a-pos"])
        out[f"amom{k}"] = np.float64(c.header["a-mom"])
        out[f"hdr{k}"] = np.array(sorted(f"{a}={b}" for a, b in c.header.items()))
        # the `cic` tool on this snapshot (src/cic/main.cc): Eulerian factor f, sub-sampling s
        for f, sub in CIC_CASES:
            subprocess.run([exe, "cic", "-i", name, "-m", k, "-f", str(f), "-s", str(sub)], cwd=work, check=True,
                           stdout=subprocess.DEVNULL)
            r = ConanFile.read(str(Path(work) / f"{name}.rho.{k}.conan"))
            out[f"rho{k}_f{f}_s{sub}"] = r.records["density"]
            out[f"rhohdr{k}_f{f}_s{sub}"] = np.array(sorted(f"{a}={b}" for a, b in r.header.items()))
    return out, snaps


def kernel_goldens():
    R = ctypes.CDLL(str(REF / "libconan_ref.so"))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    out = {}
    rng = np.random.default_rng(2024)
    for dim, N, L in [(2, 16, 10.0), (3, 8, 5.0), (1, 32, 7.0)]:
        X = rng.uniform(-1.3 * L, 2.2 * L, size=(300, dim))
        res = np.empty(N ** dim)
        R.ref_md_cic(dim, N, ctypes.c_double(L), P(X), ctypes.c_size_t(300), ctypes.c_double(1.0), P(res))
        phi = np.sin(np.arange(N ** dim) * 0.731) + 0.1 * np.cos(np.arange(N ** dim) * 0.17)
        grad = np.empty_like(X)
        R.ref_interp_gradient(dim, N, ctypes.c_double(L), P(phi), P(X), ctypes.c_size_t(300), P(grad))
        out[f"X_{dim}d"] = X
        out[f"cic_{dim}d"] = res
        out[f"phi_{dim}d"] = phi
        out[f"interp_{dim}d"] = grad
    np.savez_compressed(HERE / "kernels.npz", **out)


# (case, snapshot, linking length in units of the lattice spacing L / N) of
# the `fof` runs; the snapshots are the committed ones in <case>.npz, or for
# the 3D case made here (FOF_3D) the reference's own ic + run, kept in fof.npz
FOF_CASES = [("c1s", "2", 0.2), ("c1s", "2", 0.5), ("c1s", "2", 1.0), ("c4s", "1", 0.4), ("f3s", "2", 0.2),
             ("f3s", "2", 0.5), ("f3s", "2", 1.1)]
FOF_3D = ("f3s", "-d 3 -b 4 -L 20 --scale-free -n -1 --potential --seed 5", "-f 1 -a0 0.02 -da 0.049 -n 20")


def fof_goldens():
    """The reference's `fof` text output (src/fof/fof.cc:231-279) on committed snapshots."""
    exe = str(REF / "conan_ref")
    out = {}
    work = tempfile.mkdtemp()
    try:
        name3, ica, runa = FOF_3D
        snaps3, _ = run_cli(name3, ica, runa, work)
        for k in ("pos2", "mom2", "hdr2"):
            out[f"{name3}_{k}"] = snaps3[k]
        for name, snap, llf in FOF_CASES:
            z = {f"{a}{snap}": out[f"{name}_{a}{snap}"] for a in ("pos", "mom", "hdr")} if name == name3 \
                else np.load(HERE / f"{name}.npz")
            hdr = dict(x.split("=", 1) for x in z[f"hdr{snap}"])
            c = ConanFile(header=hdr, history=[(1700000000, "ran nbody")])
            c.add("pos", z[f"pos{snap}"])
            c.add("mom", z[f"mom{snap}"])
            src = Path(work) / f"{name}.snap.conan"
            c.write(str(src))
            ll = repr(llf * float(hdr["L"]) / int(hdr["N"]))
            key = f"{name}_{snap}_ll{llf}"
            subprocess.run([exe, "fof", "-f", str(src), "-i", key, "-l", ll], cwd=work, check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            txt = (Path(work) / f"{key}.fof.10000.txt").read_text()
            out[f"{key}_text"] = np.array(txt)
            out[f"{key}_ll"] = np.array(ll)
            out[f"{key}_L"] = np.float64(hdr["L"])
            out[f"{key}_dim"] = np.int64(hdr["dim"])
            out[f"{key}_snapshot"] = np.array(f"{name}_pos{snap}" if name == name3 else f"{name}.npz:pos{snap}")
    finally:
        shutil.rmtree(work)
    np.savez_compressed(HERE / "fof.npz", cases=np.array([f"{n}_{s}_ll{f}" for n, s, f in FOF_CASES]), **out)


def main():
    if not (REF / "conan_ref").exists():
        src = os.environ.get("CONAN_REFERENCE_SRC")
        if not src:
            raise SystemExit("oracle/_ref/conan_ref is not built: set CONAN_REFERENCE_SRC to the reference's src/")
        subprocess.run(["make", "-C", str(ROOT / "oracle"), f"REF={src}"], check=True)
    if sys.argv[1:] == ["fof"]:
        fof_goldens()
        print("fof fixtures written to", HERE)
        return
    work = tempfile.mkdtemp()
    try:
        for name, (ica, runa) in CASES.items():
            out, snaps = run_cli(name, ica, runa, work)
            np.savez_compressed(HERE / f"{name}.npz", ic_args=ica, run_args=runa, **out)
        # two reference-written files kept verbatim for the format tests
        shutil.copy(Path(work) / "c1s.density.init.conan", HERE / "c1s.density.init.conan")
        shutil.copy(Path(work) / "c3s.pos.1.conan", HERE / "c3s.pos.1.conan")
    finally:
        shutil.rmtree(work)
    kernel_goldens()
    fof_goldens()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
