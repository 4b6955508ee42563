"""Writes a generated J-scheme problem in the reference's file formats.

Record layouts (all little-endian Fortran unformatted sequential files):

``.tri`` (src/NuOpd/NuOpd.f90:678-680, read at src/NuLnz/NuCoreX.f90:838-867)
    R1  no_spart, min_cJ2, max_cJ2, proton(L4), neutron(L4), x(R4), Tparity, op(char4), del_cJ2
    R2  nJT(no_spart, min_cJ2/2:max_cJ2/2)                     int32, partition fastest
    R3  spart(no_spart): 32 x int16 shell occupations each (ptdim = 32, NuCommon.f90:17-30,203-206)
``.trd`` (NuOpd.f90:484-494, read at NuCoreX.f90:1145-1206)
    R1  trdd, 2*max_sj2, no_Opd, words, no_spartr, no_spart, op(char4)
    R2  keys(trdd)  char*8 = (2Jl, 2Jr, shell_l, shell_r, 2lam, 0, 0, 0), sorted as byte strings
    R3  dims(trdd)  int32 number of values per key
    per key with dims > 0:
      values  R4, for each right partition r, each left partition l with bit l of mask(r):
              nJT(l,Jl) x nJT(r,Jr) column-major (left state fastest)   (NuOpd.f90:328-344, 506-519)
      masks   int32 lword(1:words) for r = 1..no_spart, bit (l-1) set when block (l, r) is stored
``.oph`` (src/NuOp/NuOp.f90:410-416, read at NuCoreX.f90:1133-1142)
    R1  max_op, max_lmo;  then max_op records  opn(char8), meV(R8), pl(int32), pr(int32)
``.spe`` text: SPEs / renorm / no_level [/ restart]   (NuCoreX.f90:1664-1670)
``.sgt`` / ``.mat`` per J and species (src/NuOrth/NuOrth.f90:218-223, read at NuCoreX.f90:1216-1319)
    both start with a record holding no_spart (src/NuCommon/NuModules.F90:255-289);
    .sgt R2  num_seg, mat_dim, x(R4)
    .mat     num_seg records  dimpt, dimptr, np, npr, M(dimptr, dimpt) R4, offset(np), offset(npr),
             shell occupations of np (int16 x no_shells); segments with npr >= np in (np, npr) order.
File names of .sgt/.mat: <nucleus><file_code(J, T, nmp/2 + 36)><xtra>.<ext> (NuModules.F90:22-35).
"""
import json
import os
import numpy as np

from .fortio import RecordWriter, i4, r4, r8, l4

AN_CODE = ("0123456789_$cdefghijklmnopqrstuvwxyz@ABCDEFGHIJKLMNMPQRSTUVWXYZ" + "\xa3" + "a%^&=b-+#")
MAX_CODE = 72
X_STAMP = 1.0


def _ftrunc_div2(n):
    """Fortran integer division by 2 (truncation toward zero)."""
    return int(n / 2) if n >= 0 else -((-n) // 2)


def file_code(i, j, k):
    """src/NuCommon/NuModules.F90:22-35."""
    i = i + MAX_CODE if i < 0 else i
    j = j + MAX_CODE if j < 0 else j
    k = k + MAX_CODE if k < 0 else k
    return AN_CODE[i] + AN_CODE[j] + AN_CODE[k]


def _key(J2l, J2r, sl, sr, lam):
    return bytes([J2l, J2r, sl, sr, lam, 0, 0, 0])


def _spart(S):
    arr = np.zeros((len(S.parts), 32), dtype="<i2")
    for ip, occ in enumerate(S.parts):
        for o, k in enumerate(occ):
            arr[ip, S.shell_offset + o] = k
    return arr


def write_tri(path, S, is_proton):
    nj = (S.maxJ2 - S.minJ2) // 2 + 1
    with RecordWriter(path) as w:
        w.write(i4(len(S.parts), S.minJ2, S.maxJ2), l4(is_proton), l4(not is_proton), r4(X_STAMP),
                i4(0), b"a+a-", i4(2))
        # nJT(partition, J/2) indexed from min_cJ2/2: column-major, partition fastest
        njt = np.zeros((nj, len(S.parts)), dtype="<i4")
        for ip in range(len(S.parts)):
            for k in range(nj):
                njt[k, ip] = S.njt(ip, S.minJ2 + 2 * k)
        w.write(njt)
        w.write(_spart(S))


def density_arrays(S, rho):
    """The .trd content of species S as arrays: sorted 8-byte keys, value offsets,
    FP64 values in .trd order, and the [key][partition][word] bitmasks."""
    nsp = len(S.parts)
    words = (nsp - 1) // 32 + 1
    keys = []
    for (J2l, J2r, l, r, lam) in rho:
        keys.append((_key(J2l, J2r, S.shell_offset + l + 1, S.shell_offset + r + 1, lam), (J2l, J2r, l, r, lam)))
    keys.sort()
    vals, masks, off = [], [], [0]
    for kb, k in keys:
        blocks = rho[k]
        m = np.zeros((nsp, words), dtype=np.uint32)
        n = 0
        for ipr in range(nsp):
            for ipl in range(nsp):
                blk = blocks.get((ipl, ipr))
                if blk is None:
                    continue
                v = np.asarray(blk, dtype=np.float64).ravel(order="F")
                vals.append(v)
                n += len(v)
                m[ipr, ipl // 32] |= np.uint32(1 << (ipl % 32))
        masks.append(m)
        off.append(off[-1] + n)
    return {
        "keys": np.frombuffer(b"".join(kb for kb, _ in keys), dtype=np.uint8).copy(),
        "val_off": np.array(off, dtype=np.int64),
        "vals": np.concatenate(vals) if vals else np.zeros(0),
        "masks": np.array(masks, dtype=np.uint32).reshape(len(keys), nsp, words),
        "words": words,
    }


def segment_arrays(S, segs):
    """The .mat content of species S as arrays (segments with npr >= np, 1-based partitions;
    each segment stored as matrix(dimptr, dimpt) column-major = M^T for M = <np|H|npr>)."""
    J2s, nps, nprs, off, vals = [], [], [], [0], []
    for J2 in sorted(segs):
        for ipl, ipr, M in sorted(segs[J2], key=lambda t: (t[0], t[1])):
            J2s.append(J2)
            nps.append(ipl + 1)
            nprs.append(ipr + 1)
            v = np.asarray(M.T, dtype=np.float64).ravel(order="F")
            vals.append(v)
            off.append(off[-1] + len(v))
    return {
        "J2": np.array(J2s, dtype=np.int32), "np": np.array(nps, dtype=np.int32),
        "npr": np.array(nprs, dtype=np.int32), "off": np.array(off, dtype=np.int64),
        "vals": np.concatenate(vals) if vals else np.zeros(0),
    }


def write_trd(path, S, rho, max_j2):
    d = density_arrays(S, rho)
    nsp = len(S.parts)
    nk = len(d["val_off"]) - 1
    dims = np.diff(d["val_off"]).astype("<i4")
    with RecordWriter(path) as w:
        w.write(i4(nk, max_j2, int(d["val_off"][-1]), d["words"], nsp, nsp), b"a+a-")
        w.write(d["keys"].tobytes())
        w.write(dims)
        for k in range(nk):
            if dims[k]:
                w.write(d["vals"][d["val_off"][k]:d["val_off"][k + 1]].astype("<f4"))
                w.write(d["masks"][k].astype("<u4").view("<i4"))


def write_oph(path, vlam, norb, parity=None):
    """The pn multipole file; pl / pr are the parities of the operator's two orbit pairs
    (p1*p3 and p2*p4, src/NuOp/NuOp.f90:378-379); parity: +1/-1 per orbit (all +1 if None)."""
    par = parity if parity is not None else [1] * norb
    recs = []
    max_lmo = 0
    # both species orders, as NuOp writes them (pnnp = 0 and 1, NuOp.f90:240-262)
    for (o1, o3, o2, o4, lam), v in vlam.items():
        max_lmo = max(max_lmo, lam)
        pl, pr = par[o1] * par[o3], par[o2] * par[o4]
        recs.append((bytes([o1 + 1, o3 + 1, norb + o2 + 1, norb + o4 + 1, lam, 0, 0, 0]), v, pl, pr))
        recs.append((bytes([norb + o1 + 1, norb + o3 + 1, o2 + 1, o4 + 1, lam, 0, 0, 0]), v, pl, pr))
    recs.sort()
    with RecordWriter(path) as w:
        w.write(i4(len(recs), max_lmo))
        for kb, v, pl, pr in recs:
            w.write(kb, r8(v), i4(pl), i4(pr))


def write_spe(path, spe, renorm, no_level, restart=None):
    with open(path, "w") as f:
        f.write(" ".join(f"{x:.6f}" for x in spe) + "\n")
        f.write(f"{renorm:.6f}\n")
        f.write(f"{no_level}\n")
        if restart is not None:
            f.write(f"{restart}\n")


def like_file_names(nucleus, S, nmp, xtra):
    out = {}
    for J2 in range(S.minJ2, S.maxJ2 + 1, 2):
        out[J2] = nucleus + file_code(J2 // 2, S.n // 2, _ftrunc_div2(nmp) + MAX_CODE // 2) + xtra
    return out


def write_like(prefix_for_J, S, segs):
    for J2, base in prefix_for_J.items():
        lst = sorted(segs.get(J2, []), key=lambda t: (t[0], t[1]))
        offs = np.cumsum([0] + [S.njt(ip, J2) for ip in range(len(S.parts))])
        sp = _spart(S)
        with RecordWriter(base + ".mat") as w:
            w.write(i4(len(S.parts)))
            for ipl, ipr, M in lst:
                dimpt, dimptr = M.shape  # M = <ipl|H|ipr>: stored as matrix(dimptr, dimpt)
                w.write(i4(dimpt, dimptr, ipl + 1, ipr + 1), np.asarray(M.T, dtype="<f4").ravel(order="F"),
                        i4(offs[ipl], offs[ipr]), sp[ipl, :S.shell_offset + S.norb].copy())
        with RecordWriter(base + ".sgt") as w:
            w.write(i4(len(S.parts)))
            w.write(i4(len(lst), S.dimJ(J2)), r4(X_STAMP))


def _orbit_l(j2, parity):
    """Orbital l of an orbit from 2j and its parity (-1)^l."""
    lo = (j2 - 1) // 2
    return lo if (1 if lo % 2 == 0 else -1) == parity else lo + 1


def write_nus(path, P, nucleus):
    """The model-space file NuLnz reads first (its reader: src/NuCommon/NuCommon.f90:2546-2736),
    for the pn formalism: nucleus name, description, valence protons and neutrons, parity, the
    shells (proton shells then neutron shells: number, n, l, 2j, 2t, parity), the 2J range (one
    J here: the file is the per-J one that NuShellX's driver passes as NucleusJ), the 2T range
    with nmp, the M-scheme truncation limits (none) and output control."""
    sp = P.space
    norb = sp.norb
    lines = ["! model space of one J (written by the generator)", f"{nucleus:>6s}",
             "synthetic interaction", "pn formalism", "one J", "! valence protons, neutrons",
             f"{P.A.n} {P.B.n}", "! parity", f"{P.parity}", "! shells", f"{2 * norb}",
             "p" * norb + "n" * norb]
    for half in range(2):
        for o in range(norb):
            l = _orbit_l(sp.j2[o], sp.parity[o])
            lines.append(f"{half * norb + o + 1} {0} {l} {sp.j2[o]} 1 {sp.parity[o]}")
    tz2 = P.B.n - P.A.n
    lines += ["! 2J range", f"{P.J2} {P.J2}", "! 2T range, nmp", f"{abs(tz2)} {P.A.n + P.B.n} {tz2}",
              "! M-scheme truncation", "0 999",
              " ".join(["0"] * (2 * norb)), " ".join(str(sp.j2[o % norb] + 1) for o in range(2 * norb)),
              " ".join(["0"] * (2 * norb)), " ".join(str(sp.j2[o % norb] + 1) for o in range(2 * norb)),
              "! output control", "1"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


ANCODE = "0123456789_$cdefghijklmnopqrstuvwxyz@ABCDEFGHIJKLMNMPQRSTUVWXYZ"


def write_problem(P, outdir, tag, no_level=10, dop_cut=None, restart=None):
    """Write all input files of problem P under outdir; returns the manifest dict.  The names
    follow NuShellX's command line for the Lanczos step (src/NuShellX/NuShellx.f90:1060-1061):
    <tag><J code>.nus, <tag>a / <tag>b (.tri .trd and the like-particle .sgt/.mat), <tag>x
    (.oph .spe); manifest["args"] is that command's five arguments.  With dop_cut = (cut, cutm)
    also the compressed interaction <tag>x.dop of NuDiop (gen/dop.py); restart is the optional
    fourth line of the .spe file."""
    os.makedirs(outdir, exist_ok=True)
    A, B = P.A, P.B
    norb = P.space.norb
    base = os.path.join(outdir, tag)
    write_tri(base + "a.tri", A, True)
    write_trd(base + "a.trd", A, P.rhoA, 2 * max(P.space.j2))
    write_tri(base + "b.tri", B, False)
    write_trd(base + "b.trd", B, P.rhoB, 2 * max(P.space.j2))
    write_oph(base + "x.oph", P.vlam, norb, P.space.parity)
    write_spe(base + "x.spe", P.space.spe, P.renorm, no_level, restart)
    nus = base + ANCODE[P.J2 // 2]
    write_nus(nus + ".nus", P, tag[-6:])
    la = like_file_names(base + "a", A, -A.n, "x")
    lb = like_file_names(base + "b", B, B.n, "x")
    write_like(la, A, P.segA)
    write_like(lb, B, P.segB)
    man = {
        "a": base + "a", "b": base + "b", "int": base + "x", "like_a": base + "a", "like_b": base + "b",
        "args": [nus, base + "a", base + "b", base + "x", tag], "nucleus": tag[-6:],
        "J2": P.J2, "parity": P.parity, "nprot": A.n, "nneut": B.n, "norb": norb,
        "shell_parity": list(P.space.parity) * 2,
        "no_state": P.no_state, "nblocks": len(P.blocks),
    }
    if dop_cut is not None:
        from .dop import diop, write_dop
        write_dop(base + "x.dop", diop(P.vlam, P.space, *dop_cut))
        man["dop"] = base + "x.dop"
    with open(base + ".json", "w") as f:
        json.dump(man, f, indent=1)
    return man
