"""Constants of the flat element table, read from ``csrc/atb_table.h``.

The header is the single definition shared by the CUDA kernel and this host
compiler; parsing it here keeps the two from drifting apart.
"""
from __future__ import annotations

import os
import re

_HEADER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "atb_table.h")


def _parse(path: str) -> dict[str, int]:
    consts: dict[str, int] = {}
    pat = re.compile(r"^#define\s+(ATB_\w+)\s+(.+?)\s*(/\*.*)?$")
    with open(path) as f:
        for line in f:
            m = pat.match(line.strip())
            if not m:
                continue
            name, expr = m.group(1), m.group(2).strip()
            if name == "ATB_TABLE_H":
                continue
            expr = re.sub(r"\b(0x[0-9a-fA-F]+|\d+)u\b", r"\1", expr)
            expr = re.sub(r"\b(ATB_\w+)\b", lambda mm: str(consts[mm.group(1)]), expr)
            consts[name] = int(eval(expr, {"__builtins__": {}}))
    return consts


C = _parse(_HEADER)
globals().update(C)

#: PassMethod name -> opcode (the PassMethods on the accelerated path)
PASS_OPCODES = {
    "IdentityPass": C["ATB_OP_IDENTITY"],
    "DriftPass": C["ATB_OP_DRIFT"],
    "StrMPoleSymplectic4Pass": C["ATB_OP_STRMPOLE"],
    "StrMPoleSymplectic4RadPass": C["ATB_OP_STRMPOLE_RAD"],
    "BndMPoleSymplectic4Pass": C["ATB_OP_BNDMPOLE"],
    "BndMPoleSymplectic4RadPass": C["ATB_OP_BNDMPOLE_RAD"],
    "ThinMPolePass": C["ATB_OP_THINMPOLE"],
    "RFCavityPass": C["ATB_OP_RFCAVITY"],
    "CorrectorPass": C["ATB_OP_CORRECTOR"],
    "AperturePass": C["ATB_OP_APERTURE"],
    "QuantDiffPass": C["ATB_OP_QUANTDIFF"],
}
OPCODE_NAMES = {v: k for k, v in PASS_OPCODES.items()}
