"""Reader and writer of the HPU test-vector text files, so that key material and
ciphertexts produced for (or by) the reference's RTL flow can be fed to the
engine and the engine's outputs handed back in the same form.

Format (the reference's generator, sw/bin/gtv, as decoded against its runs):
sections start with a line "# <Name><index>"; each data line holds 512 bits
as hex, words packed from the right (word 0 in the last hex digits), and the
last line of a section is padded on the left with 'X'.

Layouts:
  ksk_hwo_<pc>.dat   u32, index (x*(k*N) + y)*L + z  -- the engine's KSK layout
                     (one AXI channel, lbx = lby = lbz = 1)
  glwe_sd_rev.dat    u64, mask polynomial then body, coefficients in
                     bit-reversed order                -> natural order here
  *_blwe_sd_rev.dat  u64, BLWE mask in natural order, body last
  inner_slwe*.dat    u32, LWE mask then body (after the key switch)

The BSK file (bsk_nd_hwo_<pc>.dat) is in the generator's network-NTT domain,
which is not decoded; keys for the engine come from luthe_keygen or from a
standard-domain BSK over Z_p.
"""
import re

import numpy as np

LINE_BITS = 512


def read_sections(path, width):
    """{section name: np.ndarray of uint32/uint64} for `width` = 32 or 64."""
    nh = width // 4
    secs, cur = {}, None
    for line in open(path):
        line = line.strip()
        if not line:
            continue
        if line.startswith("#"):
            cur = line[1:].strip()
            secs[cur] = []
            continue
        if cur is None:
            cur = ""
            secs[cur] = []
        words = [line[i:i + nh] for i in range(0, len(line), nh)][::-1]
        secs[cur].extend(int(x, 16) for x in words if "X" not in x)
    dt = np.uint64 if width == 64 else np.uint32
    return {k: np.array(v, dtype=dt) for k, v in secs.items()}


def _ordered(secs):
    """Section arrays ordered by the index at the end of their names."""
    def key(name):
        m = re.search(r"(\d+)$", name)
        return int(m.group(1)) if m else -1
    return [secs[k] for k in sorted(secs, key=key)]


def load_ksk(path):
    """KSK words in the engine's upload layout (luthe_upload_ksk)."""
    secs = read_sections(path, 32)
    if len(secs) != 1:
        raise ValueError(f"{path}: expected one section, found {len(secs)}")
    return next(iter(secs.values()))


def load_blwes(path):
    """BLWE ciphertexts, [count][k*N + 1] uint64 (mask natural, body last)."""
    return np.stack(_ordered(read_sections(path, 64)))


def load_slwes(path, width=32):
    """Key-switched LWE ciphertexts, [count][n + 1]."""
    return np.stack(_ordered(read_sections(path, width)))


def load_glwes(path, N):
    """LUT GLWEs, [count][2*N] uint64 in natural coefficient order (the
    engine's luthe_upload_luts layout)."""
    bits = N.bit_length() - 1
    rev = np.array([int(format(j, f"0{bits}b")[::-1], 2) for j in range(N)])
    out = []
    for g in _ordered(read_sections(path, 64)):
        if g.size != 2 * N:
            raise ValueError(f"{path}: GLWE of {g.size} words, expected {2 * N}")
        nat = np.empty_like(g)
        for part in range(2):
            nat[part * N + rev] = g[part * N:(part + 1) * N]
        out.append(nat)
    return np.stack(out)


def format_sections(arrays, name, width=64):
    """Text of `arrays` (one per section, sections "<name><i>") in the format
    read above."""
    nh, per = width // 4, LINE_BITS // width
    lines = []
    for i, a in enumerate(arrays):
        lines.append(f"# {name}{i}")
        vals = [int(v) for v in np.asarray(a).ravel()]
        for s in range(0, len(vals), per):
            chunk = [format(v, f"0{nh}x") for v in vals[s:s + per]]
            chunk += ["X" * nh] * (per - len(chunk))
            lines.append("".join(chunk[::-1]))
    return "\n".join(lines) + "\n"


def write_blwes(path, blwes, name="BLwe"):
    """Write BLWE ciphertexts ([count][k*N + 1] uint64) as a *_blwe_sd_rev file."""
    with open(path, "w") as f:
        f.write(format_sections(blwes, name, 64))
