"""Generate the remap golden fixtures from the reference's own test data.

Reads (only when run by hand, in a container that holds the reference tree)
the reference's `tests/golden/s003_small/` files:
  * 0001.jpg / port3_0000.tif: the reference's identity remap golden (frame 0
    of `align_image_stack_zig -m -a`), whose RGB equals the decoded JPEG and
    whose alpha is 255 everywhere;
  * 0002.jpg / port3_0001.tif / port_pair_m.pto: a real non-identity pose
    (image line 2 of the PTO) and the reference's remap of the same frame
    from a three-frame solve (compared loosely, NRMSE <= 0.005, as the
    reference's golden test does at src/golden_tests.zig:56-94).

Only row bands are stored, to keep the fixture small; the tests rebuild
full-size 768x512 sources (zeros outside the band) so the pose centres are
the reference's.  Output: tests/golden/s003_small_bands.npz.

Usage: python tests/golden/make_golden.py [reference_root]
"""
import math
import os
import sys

import numpy as np
from PIL import Image

ROOT = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
SRC = os.path.join(ROOT, "tests", "golden", "s003_small")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "s003_small_bands.npz")


def parse_pto_image_pose(path, index):
    """Pose of PTO image line `index` as ImagePose fields (src/parity_pto.zig:97-260)."""
    pano_hfov = None
    images = []
    with open(path) as fh:
        for line in fh:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "p":
                for t in tok[1:]:
                    if t.startswith("v"):
                        pano_hfov = float(t[1:])
            if tok[0] == "i":
                vals = {}
                for t in tok[1:]:
                    for key in ("TrX", "TrY", "TrZ", "Tpy", "Tpp"):
                        if t.startswith(key):
                            vals[key] = float(t[len(key):])
                            break
                    else:
                        if t[0] in "vyprabcde" and not t.startswith("n"):
                            try:
                                vals[t[0]] = float(t[1:])
                            except ValueError:
                                pass
                images.append(vals)
    v = images[index]
    deg = math.pi / 180.0
    return {
        "yaw": v["y"] * deg, "pitch": v["p"] * deg, "roll": v["r"] * deg,
        "hfov_delta": v["v"] - pano_hfov, "base_hfov_degrees": pano_hfov,
    }


def main():
    f1 = np.array(Image.open(os.path.join(SRC, "0001.jpg")).convert("RGB"))
    g0 = np.array(Image.open(os.path.join(SRC, "port3_0000.tif")))
    f2 = np.array(Image.open(os.path.join(SRC, "0002.jpg")).convert("RGB"))
    g1 = np.array(Image.open(os.path.join(SRC, "port3_0001.tif")))
    pose = parse_pto_image_pose(os.path.join(SRC, "port_pair_m.pto"), 1)
    assert f1.shape == (512, 768, 3) and g0.shape == (512, 768, 4)
    ident_rows = (0, 48)          # top border rows included
    pose_src_rows = (150, 362)    # source band around the compared rows
    pose_out_rows = (160, 352)
    np.savez_compressed(
        OUT,
        width=768, height=512,
        ident_rows=np.array(ident_rows), ident_src=f1[ident_rows[0]:ident_rows[1]],
        ident_golden=g0[ident_rows[0]:ident_rows[1]],
        ident_alpha_all_255=np.array(bool((g0[..., 3] == 255).all())),
        ident_rgb_equals_jpeg=np.array(bool(np.array_equal(g0[..., :3], f1))),
        pose_values=np.array([pose[k] for k in ("yaw", "pitch", "roll", "hfov_delta", "base_hfov_degrees")]),
        pose_src_rows=np.array(pose_src_rows), pose_src=f2[pose_src_rows[0]:pose_src_rows[1]],
        pose_out_rows=np.array(pose_out_rows), pose_golden=g1[pose_out_rows[0]:pose_out_rows[1]],
    )
    print("wrote", OUT, os.path.getsize(OUT), "bytes; pose", pose)


if __name__ == "__main__":
    main()
