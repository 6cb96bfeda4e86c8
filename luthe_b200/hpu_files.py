"""Reader and writer of the HPU test-vector text files, so that key material and
ciphertexts produced for (or by) the reference's RTL flow can be fed to the
engine and the engine's outputs handed back in the same form.

Format (the reference's generator, sw/bin/gtv, as decoded against its runs):
sections start with a line "# <Name><index>"; each data line holds 512 bits
as hex, words packed from the right (word 0 in the last hex digits), and the
last line of a section is padded on the left with 'X'.  A path ending in
".gz" is read through gzip.

Coefficient order.  The generator's "*_rev" files store polynomial
coefficients -- and the masks of BLWE ciphertexts, which are extracted from
polynomials -- in bit-reversed order: file position y holds coefficient
brv(y) of the natural order.  The engine works in natural order (its sample
extract writes natural-order masks), so the loaders below convert to natural
order unless asked for the file order, and the writer converts back.  The
KSK's mask index follows the BLWE mask, so load_ksk permutes it the same way.
A key switch gives the same result in either order as long as the KSK and
the ciphertexts agree; the blind rotation's output does not.

Layouts:
  ksk_hwo_<pc>.dat     u32, index (x*(k*N) + y)*L + z  -- the engine's KSK layout
                       (one AXI channel, lbx = lby = lbz = 1); y in file order
  bsk_nd_hwo_<pc>.dat  u64, evaluation domain over p = 2^64 - 2^32 + 1, one
                       channel: load_bsk
  glwe_sd_rev.dat      u64, mask polynomial then body, bit-reversed order
  *_blwe_sd_rev.dat    u64, BLWE mask in bit-reversed order, body last
  inner_slwe*.dat      u32, LWE mask then body (after the key switch)
"""
import re

import numpy as np

LINE_BITS = 512


def _open(path):
    path = str(path)
    if path.endswith(".gz"):
        import gzip
        return gzip.open(path, "rt")
    return open(path)


def bitrev_perm(N):
    """brv(j) for j in [0, N), N a power of two."""
    bits = N.bit_length() - 1
    return np.array([int(format(j, f"0{bits}b")[::-1], 2) if bits else 0 for j in range(N)], np.int64)


def read_sections(path, width):
    """{section name: np.ndarray of uint32/uint64} for `width` = 32 or 64."""
    nh = width // 4
    secs, cur = {}, None
    for line in _open(path):
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


def load_ksk(path, N=None, levels=None, natural=True):
    """KSK words in the engine's upload layout (luthe_upload_ksk).  With N
    (the BLWE mask size k*N) and `levels` given and natural=True, the mask
    index y is converted from the file's bit-reversed order to natural order,
    to match ciphertexts loaded with natural=True."""
    secs = read_sections(path, 32)
    if len(secs) != 1:
        raise ValueError(f"{path}: expected one section, found {len(secs)}")
    words = next(iter(secs.values()))
    if N is None or levels is None or not natural:
        return words
    return load_ksk_words_natural(words, N, levels)


def load_ksk_words_natural(words, N, levels):
    """KSK words [(n+1)][N][levels] with the mask index y permuted from the
    file's bit-reversed order to natural order (its own inverse)."""
    words = np.asarray(words)
    rows = words.size // (N * levels)
    if rows * N * levels != words.size:
        raise ValueError(f"{words.size} KSK words is not a multiple of N*levels = {N * levels}")
    k = words.reshape(rows, N, levels)
    return np.ascontiguousarray(k[:, bitrev_perm(N), :]).reshape(-1)


def blwe_file_to_natural(blwes):
    """BLWEs [count][N + 1] from the file's bit-reversed mask order to natural
    order (the permutation is its own inverse: blwe_natural_to_file is the same)."""
    b = np.asarray(blwes)
    N = b.shape[-1] - 1
    out = b.copy()
    out[..., :N] = b[..., bitrev_perm(N)]
    return out


blwe_natural_to_file = blwe_file_to_natural


def load_blwes(path, natural=True):
    """BLWE ciphertexts, [count][k*N + 1] uint64, body last; the mask in
    natural order (natural=True) or in the file's bit-reversed order."""
    b = np.stack(_ordered(read_sections(path, 64)))
    return blwe_file_to_natural(b) if natural else b


def bsk_point_order(N, psi, radix, delta):
    """k[m]: the evaluation point held by position m of a polynomial of the
    generator's bsk_nd_hwo file, m = stg_iter*(psi*radix) + p*radix + r the
    HPU's coefficient order (hw/module/hpu/simu/scripts/gen_stimuli.py:108-127:
    stg_iter, then p < psi, then r < radix).  The NTT network of the HPU
    (radix-2 pcg network, `delta` stages before it; ntt_gf64_network.py) leaves
    its last cut of d = log2(N) mod delta stages (delta if that is 0)
    bit-reversed and the rest in order: k = brv_d(m mod 2^d) * 2^(log2 N - d)
    + (m >> d).  Decoded against the generator's files for N = 64, 256 and
    2048, delta 1..7 and psi 2..32 (tests/golden/make_golden.py)."""
    if radix != 2:
        raise ValueError("only the radix-2 network is decoded")
    L = N.bit_length() - 1
    if not 1 <= delta <= L:
        raise ValueError(f"delta {delta} outside [1, {L}]")
    d = L % delta or delta
    m = np.arange(N)
    lo, hi = m & ((1 << d) - 1), m >> d
    return (bitrev_perm(1 << d)[lo] << (L - d)) | hi


PSI_4096 = 0x984EC5194D005735  # the engine's 4096-th root (psi^64 = 8)
P = 0xFFFFFFFF00000001


def _point_map(N, phi):
    """k' with phi^(2k+1) = psi_N^(2k'+1), psi_N = PSI_4096^(2048/N)."""
    psi_n = pow(PSI_4096, 2048 // N, P)
    if phi is None or phi == psi_n:
        return np.arange(N)
    x, sq = psi_n, psi_n * psi_n % P
    for u in range(1, 2 * N, 2):  # phi = psi_n^u, u odd
        if x == phi:
            k = np.arange(N)
            return ((u * (2 * k + 1)) % (2 * N) - 1) // 2
        x = x * sq % P
    raise ValueError(f"{phi:#x} is not a primitive {2 * N}-th root of unity mod p")


def load_bsk(path, n, N, psi, delta, radix=2, phi=None):
    """The generator's bsk_nd_hwo file (one channel, PBS_L = 1, k = 1) as the
    evaluation-domain BSK of luthe_upload_bsk_eval: [n][row][col][k] holding
    BSK_i[row][col](psi_N^(2k+1)) in natural k order, psi_N the engine's
    2N-th root (luthe_ntt_fwd).  `phi` is the generator's --phi-ru-2n root
    (default: psi_N, the root of the reference's simulation flow); another
    primitive 2N-th root only relabels the points.  The file's order per BR
    step i is the HPU's BSK AXI order (gen_stimuli.py:108-127): glwe_idx
    (= col, the output component), stg_iter, g_idx (= row, the decomposed
    component), p, r; the points of a polynomial follow bsk_point_order.
    `psi`, `radix` and `delta` are the generator's --psi, --ntt-radix and
    --ntt-delta."""
    words = read_sections(path, 64)
    if len(words) != 1:
        raise ValueError(f"{path}: expected one section, found {len(words)}")
    w = next(iter(words.values()))
    if w.size != n * 4 * N:
        raise ValueError(f"{path}: {w.size} words, expected n*4*N = {n * 4 * N}")
    PR = psi * radix
    if N % PR:
        raise ValueError(f"psi*radix = {PR} does not divide N = {N}")
    f = np.arange(4 * N)
    pr, row, stg, col = f % PR, (f // PR) % 2, (f // (2 * PR)) % (N // PR), f // (2 * N)
    k = _point_map(N, phi)[bsk_point_order(N, psi, radix, delta)[stg * PR + pr]]
    out = np.zeros((n, 2, 2, N), np.uint64)
    out[:, row, col, k] = w.reshape(n, 4 * N)
    return out


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


def write_blwes(path, blwes, name="BLwe", natural=True):
    """Write BLWE ciphertexts ([count][k*N + 1] uint64, mask in natural order
    unless natural=False) as a *_blwe_sd_rev file (bit-reversed mask)."""
    b = blwe_natural_to_file(blwes) if natural else np.asarray(blwes)
    with open(path, "w") as f:
        f.write(format_sections(b, name, 64))
