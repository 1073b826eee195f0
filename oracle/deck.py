"""Oracle restatement of the WanTiBEXOS stdin deck reader (test infrastructure only).

Follows ``input_read`` (subroutines/module_input_read.f90:235-663): every record is read
as two list-directed character items ``a b`` (``read(*,*,iostat=erro) a,b`` at :366);
``a`` selects the key (:369-655) and unknown keys are ignored (:652-653).  Defaults are
the values at :246-360; literals written there without a KIND suffix are single
precision, so e.g. the default KTOL is float32(0.001).
"""
from __future__ import annotations

import numpy as np


def _f32(x: float) -> float:
    return float(np.float32(x))


DEFAULTS = dict(
    nthreads=1, ngrid=[1, 1, 1], rk=0.0, nc=1, nv=1, numdos=6001.0,
    ebse0=0.0, ebsef=3.0, numbse=6001.0, sme=_f32(0.08), cshift=_f32(0.01), exc=0.0,
    mshift=[0.0, 0.0, 0.0], ktol=_f32(0.001), outputfolder="./", calcparms="./",
    meshtype="MKH", coultype="V3D", orbw="non declared file", kpaths="non declared file",
    kpathsbse="non declared file", params="", bandscalc=False, doscalc=False, bse=False,
    bsepol=False, bsekpath=False, spdiel=False, spdielpol=False, sppolbz=False, spec=False,
    berryk=False, berrybz=False, pponly=False, bsewf=False, tmcoef=False, dtfull=False,
    cpol=False, excwf0=1, excwff=2, sysdim="3D", dft="V", ta="FA", bset=False,
    bsetbnd=False, renorm=True, ediel=[1.0, 1.0, 1.0], ez=1.0, w=0.0, lc=1.0, r0=1.0,
    st=0.0, phavg=0.0, temp=0.0, pce=False, ses="AM15G", ctemp=_f32(298.15),
    tmax=_f32(5e-6), eg=0.0, egd=0.0, egs=0.0, ebgs=0.0,
)


def _split_list_directed(line: str) -> list:
    """Tokenise one record for list-directed input of character items.

    Quoted items keep inner blanks; unquoted items end at a blank or comma."""
    toks = []
    i, n = 0, len(line)
    while i < n:
        c = line[i]
        if c in " \t,":
            i += 1
            continue
        if c in "'\"":
            j = line.find(c, i + 1)
            if j < 0:
                j = n
            toks.append(line[i + 1:j])
            i = j + 1
            continue
        j = i
        while j < n and line[j] not in " \t,":
            j += 1
        toks.append(line[i:j])
        i = j
    return toks


def _logical(s: str) -> bool:
    s = s.strip().lstrip(".").upper()
    if not s:
        raise ValueError("empty logical")
    if s[0] == "T":
        return True
    if s[0] == "F":
        return False
    raise ValueError(f"bad logical {s!r}")


def _num(s: str) -> float:
    return float(s.replace("d", "e").replace("D", "E"))


_REAL = {"CTEMP=": "ctemp", "THMAX=": "tmax", "EG=": "eg", "EGD=": "egd", "EGS=": "egs",
         "EBGS=": "ebgs", "TEMP=": "temp", "PHAVG=": "phavg", "ST=": "st", "CSHIFT=": "cshift",
         "R_0=": "r0", "LC=": "lc", "EDIEL_Z=": "ez", "W_COUL=": "w", "RK=": "rk",
         "NEDOS=": "numdos", "ENSPECI=": "ebse0", "ENSPECF=": "ebsef", "NESPEC=": "numbse",
         "SIGMA=": "sme", "KTOL=": "ktol", "EXC_CORR=": "exc"}
_LOG = {"RNMD=": "renorm", "PCE=": "pce", "BSET=": "bset", "BSET_BND=": "bsetbnd",
        "DTDIAG=": "dtfull", "CPOL=": "cpol", "TMCOEF=": "tmcoef", "BSE_WF=": "bsewf",
        "PP_ONLY=": "pponly", "BERRY_BZ=": "berrybz", "BERRY=": "berryk", "SPEC=": "spec",
        "OPT_BZ=": "sppolbz", "DIEL=": "spdiel", "BSE_BND=": "bsekpath", "BSE=": "bse",
        "DOS=": "doscalc", "BANDS=": "bandscalc"}
_INT = {"EXC_WF_F=": "excwff", "EXC_WF_I=": "excwf0", "NBANDSC=": "nc", "NBANDSV=": "nv",
        "NTHREADS=": "nthreads"}
_STR = {"SES=": ("ses", 6), "TA=": ("ta", 2), "DFT=": ("dft", 1), "SYSDIM=": ("sysdim", 5),
        "COULOMB_POT=": ("coultype", 5), "MESH_TYPE=": ("meshtype", 70),
        "OUTPUT=": ("outputfolder", 70), "CALC_DATA=": ("calcparms", 70),
        "PARAMS_FILE=": ("params", 70), "KPATH_FILE=": ("kpaths", 70),
        "KPATH_BSE=": ("kpathsbse", 70), "ORB_W=": ("orbw", 70)}


def parse_deck(text: str) -> dict:
    """Return the input variables after reading ``text`` like ``input_read``."""
    d = {k: (list(v) if isinstance(v, list) else v) for k, v in DEFAULTS.items()}
    records = [_split_list_directed(line) for line in text.splitlines()]
    pairs = []
    r = 0
    # Each READ of two items starts on a fresh record, skips records without items,
    # takes the second item from the following records if needed, and the next READ
    # starts on the record after the one that supplied the second item.
    while r < len(records):
        while r < len(records) and not records[r]:
            r += 1
        if r >= len(records):
            break
        rec = records[r]
        if len(rec) >= 2:
            pairs.append((rec[0], rec[1]))
            r += 1
            continue
        a = rec[0]
        r += 1
        while r < len(records) and not records[r]:
            r += 1
        if r >= len(records):
            break  # end of file inside a READ: erro /= 0, loop exits
        pairs.append((a, records[r][0]))
        r += 1
    for a, b in pairs:
        if a in _REAL:
            d[_REAL[a]] = _num(b)
        elif a in _LOG:
            d[_LOG[a]] = _logical(b)
        elif a in _INT:
            d[_INT[a]] = int(_num(b))
        elif a in _STR:
            key, ln = _STR[a]
            d[key] = b[:ln]
        elif a in ("NGX=", "NGY=", "NGZ="):
            d["ngrid"]["XYZ".index(a[2])] = int(_num(b))
        elif a in ("EDIEL_T=", "EDIEL=", "EDIEL_B="):
            d["ediel"][{"EDIEL_T=": 0, "EDIEL=": 1, "EDIEL_B=": 2}[a]] = _num(b)
        elif a in ("SHIFT_1=", "SHIFT_2=", "SHIFT_3="):
            d["mshift"][int(a[6]) - 1] = _num(b)
        # default: ignored (module_input_read.f90:652-653)
    return d
