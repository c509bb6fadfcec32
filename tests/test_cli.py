"""Drop-in CLIs (klitho_tcc, klitho_socs) against the reference programs.

CPU tests: argument validation and error messages (these paths exit before
any GPU work).  GPU tests: the same command lines run through the reference
build (oracle/_ref, FFT shim + LAPACK forwarder) and through k-litho_b200/bin,
output files compared -- image.bin within 1e-5 of clear field, kernel_info.txt
format identical, kernels compared as weighted projectors.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O
from pngread import read_png

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "k-litho_b200", "bin")
REFBIN = os.path.join(REPO, "oracle", "_ref")
GOLDEN = os.path.join(REPO, "tests", "golden")


def run(exe, args, cwd, env=None):
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([exe] + [str(a) for a in args], cwd=cwd, capture_output=True, text=True,
                          env=e, timeout=600)


def compare_pngs(dref, dours, exact, close):
    for f in exact:
        assert np.array_equal(read_png(dref / f), read_png(dours / f)), f
    for f in close:
        a, b = read_png(dref / f).astype(int), read_png(dours / f).astype(int)
        assert a.shape == b.shape, f
        # the images differ by <= 1e-5: a pixel moves only where it sits on a
        # quantisation or colour-band edge
        differ = np.any(a != b, axis=-1) if a.ndim == 3 else (a != b)
        assert differ.mean() <= 0.01, (f, differ.mean())
        if f != "image_s.png":
            assert np.abs(a - b).max() <= 2, (f, np.abs(a - b).max())


def workdir(tmp_path, name):
    d = tmp_path / name
    (d / "out" / "kernels" / "png").mkdir(parents=True)
    return d


def tcc_args(Lx, msx, maskfile, srcType="Annular", NA=0.8, defocus=0.2, nk=8, srcSize=41):
    return [Lx, Lx, msx, msx, "Import", 128, 128, 0, maskfile, srcSize, srcType, 0.6, 0.9, 0.1,
            0.5, 1, 0.6, 0.2, "none", NA, defocus, nk]


@pytest.mark.parametrize("args,msg", [
    ([1, 2, 3], "Expected 23 arguments"),
    (tcc_args(256, 512, "m.bin"), "Invalid input parameters"),
    (tcc_args(256, 128, "m.bin", NA=1.2), "NA must be in the range [0, 1]"),
])
def test_tcc_cli_rejects_bad_arguments(tmp_path, args, msg):
    r = run(os.path.join(BIN, "klitho_tcc"), args, tmp_path)
    assert r.returncode == 1 and msg in r.stderr


@pytest.mark.parametrize("args,msg", [
    ([1, 2], "Expected 11 arguments"),
    ([256, 256, 300, 300, "LineSpace", 10, 10, 0, "x", "k/"], "Invalid input parameters"),
])
def test_socs_cli_rejects_bad_arguments(tmp_path, args, msg):
    r = run(os.path.join(BIN, "klitho_socs"), args, tmp_path)
    assert r.returncode == 1 and msg in r.stderr


def test_socs_cli_even_kernel_size_is_an_error(tmp_path):
    kd = tmp_path / "k"
    kd.mkdir()
    K.writeKernelInfo(str(kd / "kernel_info.txt"), 32, 33, [1.0])
    r = run(os.path.join(BIN, "klitho_socs"),
            [256, 256, 128, 128, "LineSpace", 10, 10, 0, "x", str(kd) + "/"], tmp_path)
    assert r.returncode == 1 and "Kernel size must be odd" in r.stderr


def read_kernel_dir(d):
    kx, ky, nk, sc = K.readKernelInfo(os.path.join(d, "kernel_info.txt"))
    n = kx * ky
    ks = []
    for i in range(nk):
        re = np.fromfile(os.path.join(d, f"krn_{i}_r.bin"), dtype=np.float32)
        im = np.fromfile(os.path.join(d, f"krn_{i}_i.bin"), dtype=np.float32)
        assert re.size == n and im.size == n
        ks.append(re.astype(np.complex128) + 1j * im)
    return kx, ky, np.array(ks), sc


def run_both_tcc(tmp_path, args, Lx, Ly, pngs=True):
    """Run klitho_tcc with `args` through the reference build and the drop-in;
    compare image.bin (1e-5 of clear field), the console's parameter block,
    kernel_info.txt and the kernels as weighted projectors."""
    dref, dours = workdir(tmp_path, "ref"), workdir(tmp_path, "ours")
    rr = run(os.path.join(REFBIN, "klitho_tcc"), args, dref)
    ro = run(os.path.join(BIN, "klitho_tcc"), args, dours)
    assert rr.returncode == 0, rr.stderr
    assert ro.returncode == 0, ro.stderr
    # console: same parameter block and the same TCC band
    for key in ("Nx: ", "TCC Size: ", "Number of Kernels: ", "Wavelength: ", "NA: "):
        lr = [l for l in rr.stdout.splitlines() if l.startswith(key)]
        lo = [l for l in ro.stdout.splitlines() if l.startswith(key)]
        assert lr == lo, (key, lr, lo)
    ir = np.fromfile(dref / "out" / "image.bin", dtype=np.float32)
    io = np.fromfile(dours / "out" / "image.bin", dtype=np.float32)
    assert ir.size == io.size == Lx * Ly
    assert np.abs(ir - io).max() <= 1e-5
    kxr, kyr, kr, sr = read_kernel_dir(dref / "out" / "kernels")
    kxo, kyo, ko, so = read_kernel_dir(dours / "out" / "kernels")
    assert (kxr, kyr) == (kxo, kyo) and len(sr) == len(so)
    assert np.allclose(so, sr, rtol=2e-5, atol=1e-6 * sr[0])
    # weighted projectors of the leading kernels up to the deepest cut inside
    # the kernel set where the spectrum has a gap (annular sources give
    # degenerate pairs, whose basis -- and a cut through them -- is arbitrary)
    m = max([j for j in range(1, len(sr)) if sr[j - 1] - sr[j] > 1e-3 * sr[0]] or [len(sr)])
    Vr, Vo = kr[:m].T, ko[:m].T
    Pr = (Vr * sr[None, :m].astype(np.float64)) @ Vr.conj().T
    Po = (Vo * so[None, :m].astype(np.float64)) @ Vo.conj().T
    assert np.linalg.norm(Po - Pr) / np.linalg.norm(Pr) <= 1e-5
    # kernel_info.txt: identical layout line by line, eigenvalues to print precision
    tr = (dref / "out" / "kernels" / "kernel_info.txt").read_text().splitlines()
    to = (dours / "out" / "kernels" / "kernel_info.txt").read_text().splitlines()
    assert len(tr) == len(to) and tr[:5] == to[:5]
    if pngs:
        # PNG outputs (common/file_io.cpp:7-135): identical inputs give identical pixels,
        # images and TCC planes agree to the colour-map quantisation
        compare_pngs(dref / "out", dours / "out", ["source.png", "mask.png"],
                     ["image.png", "image_s.png", "tcc_r.png", "tcc_i.png"])
        for i in range(len(so)):
            for part in ("r", "i"):  # kernel phases are arbitrary: same size, valid PNG
                a = read_png(dours / "out" / "kernels" / "png" / f"krn_{i}_{part}.png")
                assert a.shape == (kyo, kxo, 3)
    return dref, dours


@pytest.mark.gpu
def test_tcc_cli_matches_reference_program(tmp_path, ref_built):
    L, ms = 512, 256
    mask = synth.rect_mask(ms, 12, seed=21)
    mfile = tmp_path / "mask.bin"
    mask.astype(np.float32).tofile(mfile)
    run_both_tcc(tmp_path, tcc_args(L, ms, str(mfile)), L, L)


@pytest.mark.gpu
def test_tcc_cli_gram_path_matches_reference_program(tmp_path, ref_built):
    # a cross-quadrupole source of 196 points (radius 0.2, offset 0.5 on 41^2):
    # the drop-in's kernels come from the exact Gram step (Gram product on the
    # tensor cores, tridiagonal eigensolve on a thread-block cluster)
    L, ms = 512, 256
    mask = synth.rect_mask(ms, 12, seed=22)
    mfile = tmp_path / "mask.bin"
    mask.astype(np.float32).tofile(mfile)
    args = tcc_args(L, ms, str(mfile), srcType="CrossQuadrupole")
    args[13] = 0.2  # radius
    src = K.createSource(41, "CrossQuadrupole", radius=0.2, offset=0.5)
    assert O.source_point_count(src, O.outer_sigma(src)) == 196
    run_both_tcc(tmp_path, args, L, L)


# periods the reference accepts (klitho_tcc.cpp:391-429) beyond powers of two:
# factors of 5, an odd period, non-square
@pytest.mark.gpu
@pytest.mark.parametrize("Lx,Ly,ms", [(1000, 1000, 512), (2000, 2000, 1024), (1024, 999, 512)])
def test_tcc_cli_periods_match_reference(tmp_path, ref_built, Lx, Ly, ms):
    mask = synth.rect_mask(ms, int(40 * (ms / 1024) ** 2) + 4, seed=Lx + Ly)
    mfile = tmp_path / "mask.bin"
    mask.astype(np.float32).tofile(mfile)
    args = tcc_args(Lx, ms, str(mfile), nk=6)
    args[1] = Ly
    run_both_tcc(tmp_path, args, Lx, Ly, pngs=False)


# the reference's own example command lines (K-Litho-TCC/test_tcc.sh:49,
# K-Litho-SOCS/test_socs.sh:24): 2048 period, a 1024^2 imported mask (a seeded
# synthetic one stands in for the absent T1.bin), 101^2 annular source, NA 0.8,
# defocus 0.2, 3 kernels; then klitho_socs on the kernels klitho_tcc wrote and
# on the kernel directory the reference ships
@pytest.mark.gpu
def test_reference_example_command_lines(tmp_path, ref_built):
    mask = synth.rect_mask_fill(1024, seed=1, density=0.3)
    mfile = tmp_path / "T1.bin"
    mask.astype(np.float32).tofile(mfile)
    args = [2048, 2048, 1024, 1024, "Import", 128, 128, 0, str(mfile), 101, "Annular", 0.6, 0.9, 0.1,
            0.5, 1, 0.6, 0.2, "./source/src_test1_size101.bin", 0.8, 0.2, 3]
    dref, dours = run_both_tcc(tmp_path, args, 2048, 2048, pngs=False)
    for kd in (str(dref / "out" / "kernels") + "/", os.path.join(GOLDEN, "shipped_kernels") + "/"):
        sargs = [2048, 2048, 1024, 1024, "Import", 128, 128, 0, str(mfile), kd]
        sr, so = workdir(tmp_path, "sref" + str(len(kd))), workdir(tmp_path, "sours" + str(len(kd)))
        rr = run(os.path.join(REFBIN, "klitho_socs"), sargs, sr)
        ro = run(os.path.join(BIN, "klitho_socs"), sargs, so)
        assert rr.returncode == 0, rr.stderr
        assert ro.returncode == 0, ro.stderr
        ir = np.fromfile(sr / "out" / "image.bin", dtype=np.float32)
        io = np.fromfile(so / "out" / "image.bin", dtype=np.float32)
        assert np.abs(ir - io).max() <= 1e-5 * max(float(np.abs(ir).max()), 1.0)


# klitho_socs at periods only the general pipeline takes, including 4096
@pytest.mark.gpu
@pytest.mark.parametrize("Lx,Ly,ms", [(1000, 1000, 768), (2000, 2000, 1024), (4096, 4096, 2048),
                                      (1001, 999, 640)])
def test_socs_cli_periods_match_reference(tmp_path, ref_built, Lx, Ly, ms):
    mask = synth.rect_mask(ms, int(40 * (ms / 1024) ** 2) + 4, seed=Lx)
    mfile = tmp_path / "mask.bin"
    mask.astype(np.float32).tofile(mfile)
    src = K.createSource(41, "Annular", 0.6, 0.9)
    plan = K.TccPlan(src, 1.35, synth.defocus_arg(25.0), Lx, Ly, n_medium=1.44)
    krn, sc, _, _ = plan.topk(8)
    kd = str(tmp_path / "kgen")
    os.makedirs(kd)
    for i in range(8):
        krn[i].real.astype(np.float32).tofile(os.path.join(kd, f"krn_{i}_r.bin"))
        krn[i].imag.astype(np.float32).tofile(os.path.join(kd, f"krn_{i}_i.bin"))
    K.writeKernelInfo(os.path.join(kd, "kernel_info.txt"), 2 * plan.Nx + 1, 2 * plan.Ny + 1, sc)
    args = [Lx, Ly, ms, ms, "Import", 128, 128, 0, str(mfile), kd + "/"]
    dref, dours = workdir(tmp_path, "ref"), workdir(tmp_path, "ours")
    env = {"KLITHO_PNG": "0"}
    rr = run(os.path.join(REFBIN, "klitho_socs"), args, dref)
    ro = run(os.path.join(BIN, "klitho_socs"), args, dours, env=env)
    assert rr.returncode == 0, rr.stderr
    assert ro.returncode == 0, ro.stderr
    ir = np.fromfile(dref / "out" / "image.bin", dtype=np.float32)
    io = np.fromfile(dours / "out" / "image.bin", dtype=np.float32)
    assert ir.size == io.size == Lx * Ly
    assert np.abs(ir - io).max() <= 1e-5 * max(float(np.abs(ir).max()), 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("kdir", ["shipped", "generated"])
def test_socs_cli_matches_reference_program(tmp_path, ref_built, kdir):
    L, ms = 512, 384
    mask = synth.rect_mask(ms, 20, seed=5)
    mfile = tmp_path / "mask.bin"
    mask.astype(np.float32).tofile(mfile)
    if kdir == "shipped":
        kd = os.path.join(GOLDEN, "shipped_kernels")
    else:
        src = K.createSource(41, "Annular", 0.6, 0.9)
        plan = K.TccPlan(src, 1.35, synth.defocus_arg(25.0), L, L, n_medium=1.44)
        krn, sc, ev, _ = plan.topk(12)
        kd = str(tmp_path / "kgen")
        os.makedirs(kd)
        for i in range(12):
            krn[i].real.astype(np.float32).tofile(os.path.join(kd, f"krn_{i}_r.bin"))
            krn[i].imag.astype(np.float32).tofile(os.path.join(kd, f"krn_{i}_i.bin"))
        K.writeKernelInfo(os.path.join(kd, "kernel_info.txt"), 2 * plan.Nx + 1, 2 * plan.Ny + 1, sc)
    args = [L, L, ms, ms, "Import", 128, 128, 0, str(mfile), kd + "/"]
    dref, dours = workdir(tmp_path, "ref"), workdir(tmp_path, "ours")
    rr = run(os.path.join(REFBIN, "klitho_socs"), args, dref)
    ro = run(os.path.join(BIN, "klitho_socs"), args, dours)
    assert rr.returncode == 0, rr.stderr
    assert ro.returncode == 0, ro.stderr
    ir = np.fromfile(dref / "out" / "image.bin", dtype=np.float32)
    io = np.fromfile(dours / "out" / "image.bin", dtype=np.float32)
    _, _, _, sc = K.readKernelInfo(os.path.join(kd, "kernel_info.txt"))
    cf = float(np.abs(ir).max())
    assert np.abs(ir - io).max() <= 1e-5 * max(cf, 1.0)
    compare_pngs(dref / "out", dours / "out", ["mask.png"], ["image.png", "image_s.png"])
