"""Catalogue files in the reference's pipe-separated format.

The reference reads fields 0 (NORAD id), 1 (name), 2 (object type), 4
(country), 5 (radar cross-section class) and 11-16 (ECI position and velocity,
km and km/s) of every non-comment row, and the common epoch from a header line
containing "epoch commun) : YYYY-MM-DDTHH:MM:SS" (src/core/orbital.cpp:136-188).
Object sizes follow from the RCS class: SMALL 0.2 m, LARGE 4 m, other 0.8 m.
"""
import numpy as np

RCS_SIZE_M = {"SMALL": 0.2, "MEDIUM": 0.8, "LARGE": 4.0}


def rcs_class_for_size(size_m):
    """The RCS class whose reference size is closest (in log) to size_m."""
    s = np.asarray(size_m, dtype=np.float64)
    return np.where(s < 0.4, "SMALL", np.where(s < 1.8, "MEDIUM", "LARGE"))


def write_catalog(path, states, ids=None, names=None, rcs=None, epoch_iso="2026-08-01T10:00:00+00:00", types=None):
    """Writes states (n, 6) as a catalogue the reference CLI can read.

    Values are written with 17 significant digits, so they read back bit for bit.
    types: object types (PAYLOAD, DEBRIS, ROCKET BODY, UNKNOWN); DEBRIS by default.
    """
    st = np.asarray(states, dtype=np.float64)
    n = st.shape[0]
    ids = np.arange(1, n + 1) if ids is None else np.asarray(ids)
    names = [f"OBJ {int(i)}" for i in ids] if names is None else list(names)
    rcs = ["MEDIUM"] * n if rcs is None else list(rcs)
    types = ["DEBRIS"] * n if types is None else list(types)
    with open(path, "w") as f:
        f.write("# Synthetic catalogue, seeded, states at one common epoch\n")
        f.write(f"# Reference date (epoch commun) : {epoch_iso}\n")
        f.write("# Columns: NORAD_ID | NAME | OBJECT_TYPE | INTL_DES | COUNTRY | RCS_SIZE | RCS_VALUE_m2 | "
                "TLE_EPOCH | LAT_deg | LON_deg | ALT_km | X_km | Y_km | Z_km | VX_km_s | VY_km_s | VZ_km_s\n")
        for k in range(n):
            x = st[k]
            alt = float(np.linalg.norm(x[:3])) - 6378.137
            vals = " | ".join(f"{v:.17g}" for v in x)
            f.write(f"{int(ids[k])} | {names[k]} | {types[k]} | 2026-000A | XX | {rcs[k]} | 0 | "
                    f"2026-08-01T10:00:00 | 0 | 0 | {alt:.3f} | {vals}\n")


def read_catalog(path):
    """(ids, names, rcs, states) from a catalogue file (rows with >= 17 fields)."""
    ids, names, rcs, states = [], [], [], []
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            fld = [t.strip() for t in line.rstrip("\n").split("|")]
            if len(fld) < 17:
                continue
            ids.append(int(fld[0]))
            names.append(fld[1])
            rcs.append(fld[5])
            states.append([float(v) for v in fld[11:17]])
    return np.array(ids), names, rcs, np.array(states, dtype=np.float64).reshape(-1, 6)
