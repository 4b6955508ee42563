"""The reference's output files (.abz, .trl, .lev) from nsx_write_results and the nulnz_gpu
command, read back the way NuVec reads them (src/NuVec/NuVec.f90:120-131, 180-198, 210-216):
the thick-restart .abz matrix is diagonalised and its eigenvectors combine the .trl records
into the states, which must be the solver's eigenpairs.

Tolerances: the .trl records and the .abz values are FP32 (the reference's storage), so the
reconstructed states match the solver's to 1e-6 relative, the energies to FP32 rounding, and
the .lev levels to the printed 3 decimals."""
import os
import struct
import subprocess
import numpy as np
import pytest

from conftest import ROOT, make_problem, write_files



def read_records(path):
    """Fortran unformatted sequential records (4-byte length markers)."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        (n,) = struct.unpack_from("<i", data, i)
        rec = data[i + 4:i + 4 + n]
        (n2,) = struct.unpack_from("<i", data, i + 4 + n)
        assert n == n2
        out.append(rec)
        i += 8 + n
    return out


def read_outputs(prefix, S, nev):
    """(energies, states, levels, parity characters) as NuVec would reconstruct them: the lowest
    nev eigenpairs of the .abz matrix, the states as its eigenvectors times the .trl records.
    The files hold either the eigenpairs themselves (nsx_write_results: matrix = diag(E), one
    record per state) or the solver's thick-restart state (nsx_write_state: matrix = V^T H V of
    the basis, the basis records, then the next Lanczos vector)."""
    recs = read_records(prefix + ".abz")
    assert len(recs) == 4
    r1 = recs[0]
    (isave,) = struct.unpack_from("<i", r1, 0)
    assert isave >= nev and len(r1) == 4 + 4 * (2 * isave + isave * isave)
    a = np.frombuffer(r1, dtype="<f4", count=isave, offset=4)
    matrix = np.frombuffer(r1, dtype="<f4", count=isave * isave, offset=4 + 8 * isave).reshape(isave, isave,
                                                                                               order="F")
    r2 = struct.unpack("<iifiiiiiiii", recs[1])
    imax, no_level, tt, no_state, basd, count = r2[:6]
    assert no_level == nev and no_state == S.dim and basd == len(S.blocks) and count == 2
    bas = recs[2]
    assert len(bas) == 8 * basd
    for k, (ja, jb, _, _) in enumerate(S.blocks):
        assert bas[8 * k] == ja and bas[8 * k + 1] == jb and bas[8 * k + 2:8 * k + 8] == b"\0" * 6
    assert len(recs[3]) == 4 * (300 + 1 + 300)
    trl = np.fromfile(prefix + ".trl", dtype="<f4").reshape(-1, S.dim)
    assert trl.shape[0] in (isave, isave + 1)
    assert np.allclose(a, np.diag(matrix))
    w, U = np.linalg.eigh(matrix.astype(np.float64))
    w, U = w[:nev], U[:, :nev]
    psi = U.T @ trl[:isave].astype(np.float64)
    lines = open(prefix + ".lev").read().splitlines()
    k0 = next(i for i, l in enumerate(lines) if "Lowest Energy Levels" in l)
    body = "".join(l for l in lines[k0 + 1:] if l.strip())
    lv = [float(body[k:k + 10]) for k in range(0, len(body), 11)]
    return w, psi, np.array(lv), body[10::11]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sd_2p2n_0", "fp_4p4n_0"])
def test_write_results_reads_back_as_nuvec_does(name, tmp_path):
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Solver, NSX_FP64
    build()
    P = make_problem(name)
    S = Solver.from_problem(P)
    nev = 6
    ev, vecs, rep = S.solve(nev=nev, tol=1e-8, precision=NSX_FP64, want_vectors=True)
    prefix = str(tmp_path / "out")
    S.write_results(prefix, ev, vecs, rep["iterations"], "synthetic", 0)
    w, psi, lv, par = read_outputs(prefix, S, nev)
    assert np.allclose(w, ev, rtol=1e-6, atol=1e-6)
    for i in range(nev):
        s = np.sign(psi[i] @ vecs[i])
        assert np.abs(s * psi[i] - vecs[i]).max() <= 1e-6 * np.abs(vecs[i]).max()
    assert np.allclose(lv, ev, atol=6e-4)
    assert set(par) == {"+"}          # J^pi = 0+ in the positive-parity sector
    # .xvc, as NuVec writes it: (no_state, levels), then (E, vector) per level in FP32
    recs = read_records(prefix + ".xvc")
    assert struct.unpack("<ii", recs[0]) == (S.dim, nev) and len(recs) == nev + 1
    for i in range(nev):
        assert len(recs[i + 1]) == 4 * (1 + S.dim)
        e = struct.unpack_from("<f", recs[i + 1], 0)[0]
        v = np.frombuffer(recs[i + 1], dtype="<f4", offset=4)
        assert abs(e - ev[i]) <= 1e-6 * max(1.0, abs(ev[i]))
        assert np.abs(v - vecs[i]).max() <= 1e-6 * np.abs(vecs[i]).max()
    S.close()


@pytest.mark.gpu
def test_nulnz_gpu_command_writes_the_reference_outputs(files_dir):
    from nushellx_b200.build import build, CLI
    from nushellx_b200.nsx import Solver, NSX_FP64
    build()
    P = make_problem("fp_4p4n_0")
    man = write_files(P, os.path.join(files_dir, "cli44"), "cli44")
    nuc = os.path.join(files_dir, "cli44", "Fe")
    cmd = [CLI, "--a", man["a"], "--b", man["b"], "--int", man["int"], "--like-a", man["like_a"],
           "--like-b", man["like_b"], "--nprot", str(man["nprot"]), "--nneut", str(man["nneut"]),
           "--J2", str(man["J2"]), "--parity", str(man["parity"]),
           "--shell-parity", ",".join(str(p) for p in man["shell_parity"]), "--nshells-p", str(man["norb"]),
           "--nucleus", nuc]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    S = Solver.from_files(man)
    e64, _, _ = S.solve(nev=10, tol=1e-8, precision=NSX_FP64)
    from nushellx_b200.nsx import load_library
    import ctypes
    code = ctypes.create_string_buffer(4)
    load_library().nsx_file_code(man["J2"] // 2, man["nprot"], man["nneut"], code)
    prefix = nuc + code.value.decode()
    w, psi, lv, par = read_outputs(prefix, S, 10)
    assert np.abs(w - e64).max() < 1e-5                      # |dE| against the FP64 answer
    assert np.allclose(lv, e64, atol=6e-4)
    for i in range(10):                                       # the states are eigenvectors of H
        hv = S.matvec_host(psi[i], NSX_FP64)
        assert np.linalg.norm(hv - w[i] * psi[i]) <= 2e-3 * np.linalg.norm(psi[i])
    S.close()


@pytest.mark.gpu
def test_nulnz_gpu_takes_nushellx_command_line(files_dir):
    """The positional form NuShellX's driver runs (src/NuShellX/NuShellx.f90:1060-1061):
    NucleusJ Nucleus'a' Nucleus'b' Nucleus+xtra intfile, the model space from NucleusJ.nus."""
    from nushellx_b200.build import build, CLI
    from nushellx_b200.nsx import Solver, NSX_FP64, load_library
    import ctypes
    build()
    P = make_problem("sd_2p2n_2")
    d = os.path.join(files_dir, "clisd")
    man = write_files(P, d, "sd22")
    r = subprocess.run([CLI, *man["args"], "--precision", "fp64", "--tol", "1e-8"], capture_output=True, text=True,
                       timeout=600, cwd=d)
    assert r.returncode == 0, r.stderr
    code = ctypes.create_string_buffer(4)
    load_library().nsx_file_code(man["J2"] // 2, man["nprot"], man["nneut"], code)
    prefix = os.path.join(d, man["nucleus"] + code.value.decode())
    S = Solver.from_files(man)
    e64, _, _ = S.solve(nev=10, tol=1e-9, precision=NSX_FP64)
    w, psi, lv, par = read_outputs(prefix, S, 10)
    assert np.abs(w - e64).max() < 1e-6
    S.close()


@pytest.mark.parametrize("broken", ["int", "a", "nev"])
def test_nulnz_gpu_stops_with_a_message(broken, files_dir):
    """Missing files and bad arguments end the command with a message and a non-zero exit
    status, as the reference's stop does (these paths fail before any GPU call)."""
    from nushellx_b200.build import build, CLI
    build()
    P = make_problem("sd_2p2n_0")
    man = write_files(P, os.path.join(files_dir, "clierr"), "clierr")
    cmd = [CLI, "--a", man["a"], "--b", man["b"], "--int", man["int"], "--like-a", man["like_a"],
           "--like-b", man["like_b"], "--nprot", "2", "--nneut", "2", "--J2", "0", "--parity", "1",
           "--shell-parity", "1,1,1,1,1,1", "--nshells-p", "3", "--nucleus", os.path.join(files_dir, "clierr", "X")]
    if broken == "nev":
        cmd += ["--nev", "0"]
        msg = "out of range"
    else:
        cmd[cmd.index("--" + broken) + 1] += "_missing"
        cmd += ["--nev", "4"] if broken == "a" else []
        msg = "cannot open"
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and msg in r.stderr, r.stderr


@pytest.mark.gpu
def test_state_files_resume_to_the_same_eigenvalues(tmp_path):
    """The thick-restart state in the reference's TRL files (.abz matrix/counters, .trl basis and
    next vector) read back and resumed (NuCoreX.f90:266-292): the resumed solve reaches the same
    eigenvalues, and NuVec's reconstruction from the written files gives them too."""
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Solver, NSX_FP64
    build()
    P = make_problem("fp_4p4n_0")
    S = Solver.from_problem(P)
    e_ref, _, _ = S.solve(nev=6, tol=1e-9, precision=NSX_FP64)
    # a short first run: stopped by its iteration limit, as an interrupted job would be
    e1, v1, r1, st = S.solve_state(nev=6, tol=1e-9, precision=NSX_FP64, window=40, max_iter=60)
    assert r1["converged"] < 6 and st["V"].shape[0] > 6
    V = st["V"]
    assert np.abs(V @ V.T - np.eye(len(V))).max() < 1e-10
    prefix = str(tmp_path / "fe")
    S.write_state(prefix, st, e1, v1)
    st2 = S.read_state(prefix)
    assert st2["V"].shape == st["V"].shape and abs(st2["beta"] - st["beta"]) < 1e-6 * max(1.0, abs(st["beta"]))
    w, psi, lv, par = read_outputs(prefix, S, 6)     # NuVec's view of the state files
    T = st["T"]
    assert np.abs(w - np.linalg.eigvalsh(T)[:6]).max() < 1e-5
    e2, v2, r2, _ = S.solve_state(nev=6, tol=1e-9, precision=NSX_FP64, window=40, max_iter=3000, resume=st2)
    assert r2["converged"] == 6 and r2["restarts"] >= 1
    assert np.abs(e2 - e_ref).max() < 1e-8
    S.close()
