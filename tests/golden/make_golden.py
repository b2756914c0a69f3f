"""Regenerate the golden fixtures under tests/golden/ from a checkout of the
reference project (BlauHimmel/Hikari).

The pathMIS known-answer scenes are the reference's own Student-t test files
scene/pa5/tests/test-direct.xml (references 0.0898394, 0.02292, 0.0534198,
0.0205314, 0.26174) and test-furnace.xml (references 2, 5) with the OBJ files
they load.  They are copied verbatim so the tests run without the reference.

usage: python tests/golden/make_golden.py <path-to-reference-checkout>
"""
import os
import shutil
import sys

FILES = ["test-direct.xml", "test-furnace.xml", "floor.obj", "furnace.obj"] + [
    f"polylum{i}.obj" for i in range(1, 6)
]


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "scene", "pa5", "tests")
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pa5")
    os.makedirs(dst, exist_ok=True)
    for f in FILES:
        shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
        print("copied", f)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
