"""Copies the reference's scene fixtures that the tests read into
tests/golden/fixtures/ (run once where the reference checkout exists; the
copies are committed so the tests run anywhere).

The reference's tests/fixtures folder holds RIB scene files and a Radiance
sky map. The RIB files under 12 KB are copied, plus sky.hdr (their dome
lights' map). The multi-megabyte archives (forest_grass.rib,
forest_ground.rib, forest_lights.rib, kid_character.rib) and the .tex / .png
texture files are left out; scenes that name them load with a warning for
each missing file, as the reference's builder does.
"""
import os
import shutil
import sys

SRC = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/tests/fixtures"
DST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fixtures")
MAX_RIB = 12 * 1024


def main():
    os.makedirs(DST, exist_ok=True)
    for name in sorted(os.listdir(SRC)):
        path = os.path.join(SRC, name)
        keep = (name.endswith(".rib") and os.path.getsize(path) <= MAX_RIB) or name == "sky.hdr"
        if keep:
            shutil.copyfile(path, os.path.join(DST, name))
            print(name)


if __name__ == "__main__":
    main()
