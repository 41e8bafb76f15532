"""Generate the level-set golden fixtures with the reference's own DistrGen code.

Runs the functions of the reference's DistrGen/fluidLevelSets.py
(generate_solid_init, generate_fluid_with_ball_init) and
DistrGen/fluidLabels.py (generate_combined_labels_simple) at a small size and
copies their output files into tests/golden/levelsets/.  The functions are
taken from the reference sources by name (their modules also run plotting and
full-size generation at import, which is skipped).  Run from the repository
root with the reference checkout named by FLUIDPRJCT_REFERENCE:

    FLUIDPRJCT_REFERENCE=<checkout> python tests/golden/make_levelset_golden.py
"""
import ast
import os
import shutil
import sys
import tempfile

REF = os.environ.get("FLUIDPRJCT_REFERENCE", "")
if not REF:
    sys.exit("set FLUIDPRJCT_REFERENCE to the root of a reference checkout")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "levelsets")


def load_functions(path, names):
    tree = ast.parse(open(path).read(), path)
    mod = ast.Module(body=[n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names],
                     type_ignores=[])
    ns = {"os": os}
    exec(compile(mod, path, "exec"), ns)
    missing = [n for n in names if n not in ns]
    if missing:
        sys.exit(f"not found in {path}: {missing}")
    return ns


def main():
    ls = load_functions(os.path.join(REF, "DistrGen", "fluidLevelSets.py"),
                        ["generate_solid_init", "generate_fluid_with_ball_init"])
    lb = load_functions(os.path.join(REF, "DistrGen", "fluidLabels.py"), ["generate_combined_labels_simple"])
    w, h = 40, 32
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        solid = os.path.join(tmp, "res", "solid_init.txt")
        fluid = os.path.join(tmp, "res", "fluid_init_ball.txt")
        labels = os.path.join(tmp, "res", "labels_simple.txt")
        ls["generate_solid_init"](solid, w=w, h=h, wall_thickness=2, floor_thickness=3)
        ls["generate_fluid_with_ball_init"](fluid, w=w, h=h, wall_thickness=2, floor_thickness=3,
                                            fill_width_frac=0.6, fill_height_frac=0.35,
                                            ball_center_frac=(0.7, 0.3), ball_radius_frac=0.15)
        lb["generate_combined_labels_simple"](solid, fluid, labels)
        for f in (solid, fluid, labels):
            shutil.copy(f, os.path.join(OUT, os.path.basename(f)))
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
