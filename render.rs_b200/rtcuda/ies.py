"""IES photometric profiles (LM-63) for point lights, read as the
reference's ``IesProfile::parse`` does (src/scene/ies.rs:27-82): header
lines up to ``TILT=`` (only ``TILT=NONE``), then whitespace-separated
numbers: lamp count, lumens per lamp, candela multiplier, the vertical and
horizontal angle counts, six geometry / unit values, the three ballast
values, the vertical angles, the horizontal angles, and one row of
vertical candela values per horizontal angle (scaled by the multiplier).
Tokens that are not numbers are skipped, as the reference's parse does."""
import numpy as np


class IesError(ValueError):
    pass


def parse_ies(text):
    """(v_angles, h_angles, candela[h][v]) of an LM-63 profile."""
    pos = text.find("TILT=")
    if pos < 0:
        raise IesError("IES: no TILT= line")
    after = text[pos:]
    end = after.find("\n")
    end = len(after) if end < 0 else end
    tilt = after[:end].strip()
    if tilt != "TILT=NONE":
        raise IesError(f"IES: only TILT=NONE is supported (got {tilt})")
    nums = []
    for tok in after[end:].split():
        try:
            nums.append(float(tok))
        except ValueError:
            pass
    if len(nums) < 13:
        raise IesError("IES: truncated numeric block")
    n_v, n_h, mult = int(nums[3]), int(nums[4]), nums[2]
    if n_v == 0 or n_h == 0 or n_v > 4096 or n_h > 4096:
        raise IesError(f"IES: implausible angle counts {n_v}x{n_h}")
    rest = nums[13:]
    v, h = rest[:n_v], rest[n_v:n_v + n_h]
    if len(v) < n_v or len(h) < n_h:
        raise IesError("IES: missing angle values")
    c = rest[n_v + n_h:n_v + n_h + n_v * n_h]
    if len(c) < n_v * n_h:
        raise IesError("IES: missing candela values")
    return (np.array(v, np.float64), np.array(h, np.float64),
            np.array(c, np.float64).reshape(n_h, n_v) * mult)


def load_ies(path):
    with open(path, "r", errors="replace") as f:
        return parse_ies(f.read())
