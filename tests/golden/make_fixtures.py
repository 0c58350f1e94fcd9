"""Copy the reference's own golden decks into tests/golden/.

The HAMS-MREL reference ships its regression data as input decks
(ControlFile.in, .pnl meshes, Hydrostatic.in, generalized-mode files) with
the HAMS-format outputs its Fortran build produced.  The GPU box used for the
CUDA tests has no copy of the reference, so the decks the parity tests need
are committed here.  Run this script in a checkout that has the reference
next to it:

    python tests/golden/make_fixtures.py /path/to/HAMS-MREL

Decks copied (reference path -> fixture name):
  test/data/config1                       -> config1   (3 bodies x 234 panels, h = 70 m)
  examples/example2_multi_bodies_wave_fields -> example2 (10 bodies x 234, h = 14.5 m)
  examples/example5_single_body           -> example5  (1 body, 234 panels + 383 lid panels)
  examples/example3_multi_bodies_gen_mod  -> example3  (2 bodies x 234 panels with lids, a generalized
                                                        mode; its expected files hold the first of the
                                                        deck's 10 frequencies only)
Only the HAMS-format outputs (OAMASS/ODAMPING/OEXFOR) are kept as expected data, plus
the WAMIT-format force, motion and hydrostatic files of example2, example3 and example5
and example2's field-point files (PressureElevation.6p, PressureElevationIncidence.6p:
100 points on the free surface).
"""
import os
import shutil
import sys

DECKS = {
    "config1": ("test/data/config1/input", "test/data/config1/expected_output"),
    "example2": ("examples/example2_multi_bodies_wave_fields/Input",
                 "examples/example2_multi_bodies_wave_fields/Output/Hams_format"),
    "example5": ("examples/example5_single_body/Input",
                 "examples/example5_single_body/Output/Hams_format"),
    "example3": ("examples/example3_multi_bodies_gen_mod/Input",
                 "examples/example3_multi_bodies_gen_mod/Output/Hams_format"),
    "example1": ("examples/example1_multi_bodies/Input",
                 "examples/example1_multi_bodies/Output/Hams_format"),
}
# Expected files cut to their first records: example1 (5 bodies x 727 panels,
# h = 0.9 m, 0_inf_frequency_limits = 1) keeps the zero- and infinite-frequency
# limits and the first regular frequency, the part its tests rerun.
TRIM = {"example1": 3}
OUTPUTS = [f"{k}{m}.txt" for k in ("OAMASS", "ODAMPING", "OEXFOR") for m in range(1, 7)]
FORCES = ["AmssDamp.1", "ExcForce.3", "Motion.4", "Hydrostat.hst"]
WAMIT = {"example2": ("examples/example2_multi_bodies_wave_fields/Output/Wamit_format",
                      FORCES + ["PressureElevation.6p", "PressureElevationIncidence.6p"]),
         "example3": ("examples/example3_multi_bodies_gen_mod/Output/Wamit_format", FORCES),
         "example5": ("examples/example5_single_body/Output/Wamit_format", FORCES)}


def _copy_first_records(src, dst, nrec):
    """Copy the rows of the first nrec distinct (frequency column 1, 2) heads."""
    heads, out = [], []
    for line in open(src):
        key = tuple(line.split()[:2])
        if not key:
            continue
        if key not in heads:
            heads.append(key)
        if len(heads) > nrec:
            break
        out.append(line)
    with open(dst, "w") as f:
        f.writelines(out)


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for name, (inp, exp) in DECKS.items():
        dst_in = os.path.join(here, name, "input")
        dst_exp = os.path.join(here, name, "expected")
        os.makedirs(dst_in, exist_ok=True)
        os.makedirs(dst_exp, exist_ok=True)
        src_in = os.path.join(ref_root, inp)
        for f in sorted(os.listdir(src_in)):
            shutil.copyfile(os.path.join(src_in, f), os.path.join(dst_in, f))
        for f in OUTPUTS:
            src = os.path.join(ref_root, exp, f)
            if name in TRIM:
                _copy_first_records(src, os.path.join(dst_exp, f), TRIM[name])
            else:
                shutil.copyfile(src, os.path.join(dst_exp, f))
        if name in WAMIT:
            src, files = WAMIT[name]
            for f in files:
                shutil.copyfile(os.path.join(ref_root, src, f), os.path.join(dst_exp, f))
        print(f"{name}: {len(os.listdir(dst_in))} input files, {len(os.listdir(dst_exp))} expected files")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_fixtures.py <root of the HAMS-MREL source tree>")
    main(sys.argv[1])
