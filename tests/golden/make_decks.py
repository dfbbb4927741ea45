"""Copy the reference's own run decks into tests/golden/decks/ as fixtures.

    python tests/golden/make_decks.py /path/to/LBcuda

The decks (Tests/*/input.dat, the namelist deck Tests/CPC_Tab2_128/newinput.dat
of the NEWINPUT build, the small input.xyz files and the first 1280
particles of Tests/07-1280-Particle/input.xyz.256cube.5000.r5.5) are data the
reference ships for its runs; the tests parse them with the host-side input
readers and check the parser's verdicts (the stale 8-line decks 02-06 must be
rejected, main.CUF:478-493).
"""
import os
import shutil
import sys

DECKS = ["01", "02", "03", "04", "05-1Particle", "06-12_Particle", "07-1280-Particle",
         "CPC_Tab2_128", "CPC_Tab2_256"]


def main(ref):
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "decks")
    os.makedirs(out, exist_ok=True)
    for d in DECKS:
        src = os.path.join(ref, "Tests", d, "input.dat")
        shutil.copy(src, os.path.join(out, f"{d}.input.dat"))
    shutil.copy(os.path.join(ref, "Tests", "CPC_Tab2_128", "newinput.dat"),
                os.path.join(out, "CPC_Tab2_128.newinput.dat"))
    for d in ["05-1Particle", "06-12_Particle"]:
        shutil.copy(os.path.join(ref, "Tests", d, "input.xyz"), os.path.join(out, f"{d}.input.xyz"))
    for f in ["input_3a.dat", "input_3b.dat", "input_3c.dat"]:
        shutil.copy(os.path.join(ref, "Tests", "CPC_Tab3", f), os.path.join(out, f"CPC_Tab3.{f}"))
    # first 1280 spheres of the 256^3, r = 5.5 placement
    src = os.path.join(ref, "Tests", "07-1280-Particle", "input.xyz.256cube.5000.r5.5")
    with open(src) as fh:
        lines = fh.read().splitlines()
    keep = ["1280"] + lines[1:2] + lines[2:2 + 1280]
    with open(os.path.join(out, "07-1280.input.xyz.256cube.r5.5"), "w") as fh:
        fh.write("\n".join(keep) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_decks.py <LBcuda checkout>")
    main(sys.argv[1])
