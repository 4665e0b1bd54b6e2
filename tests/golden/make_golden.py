"""Extract the reference's own numeric artefacts into small fixtures.

Run where the reference tree is mounted, with its mode1_bbl directory as the
one argument:
    python tests/golden/make_golden.py <reference>/mode1_bbl
It reads text files that the reference's runs wrote and stores them as JSON
under tests/golden/.  The GPU box never reads the reference tree.

* testout.dat     -- testhelm (testhelm.f:1-134): penalty solve of
                     f - eps f'' = eps, f = 0 at both ends, eps = 1e-2,
                     10 subdomains x 25 points of runfolder/subd.dat, zlen=5.
* z_grid.dat      -- GLL grid of the shipped 12-subdomain run (setup.f:151-166)
* x_grid.dat      -- x grid (setup.f:136-142)
* uveltest.dat    -- u(32,1,10), u(32,1,50) at 16 digits (various.f:743-745):
                     rows 1041-1049, t=0..0.8 of the shipped 2-D forced run,
                     and rows 641-1040, the 400 steps of the recorded run
                     whose log is `output`
* minmaxtest.dat, cfl.dat, avgint.dat -- per-step traces of the same run
* runfolder/subd.dat, subd.dat -- subdomain tables used above
* rhomean.dat      -- setup.f:170-184 of the shipped run: z, rhomean(z),
                     rhograd, (N(z)/N)^2, fshear(z) from the top level down
* output, dtchange.dat -- the log of a recorded 400-step run (xlen = 40) and
                     its record of time-step changes (write(65,*) t, dt,
                     various.f:971): the run's parameters and wave frequency
                     (main.f:370), maxcalc's cflzmax at the start of every
                     step (various.f:882) and the (t, dt) of every change;
                     the (counter, t) of every animation dump the run logged
                     (solver.f:169-170)
"""
import json
import os
import sys


def rows(path, skip=0):
    out = []
    for line in open(path).read().splitlines()[skip:]:
        parts = line.split()
        if not parts:
            continue
        try:
            out.append([float(x.replace("D", "E")) for x in parts])
        except ValueError:
            continue
    return out


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    g = {}
    g["testout"] = [r[:2] for r in rows(os.path.join(ref, "testout.dat"), 1)]
    g["z_grid"] = rows(os.path.join(ref, "z_grid.dat"))
    g["x_grid"] = rows(os.path.join(ref, "x_grid.dat"))
    lines = open(os.path.join(ref, "uveltest.dat")).read().splitlines()
    g["uveltest"] = [[float(x) for x in l.split()] for l in lines[1040:1049]]
    g["uveltest_recorded_run"] = [[float(x) for x in l.split()] for l in lines[640:1040]]
    g["minmaxtest"] = rows(os.path.join(ref, "minmaxtest.dat"))
    g["cfl"] = rows(os.path.join(ref, "cfl.dat"), 1)
    g["avgint"] = rows(os.path.join(ref, "avgint.dat"), 1)
    g["subd_runfolder"] = rows(os.path.join(ref, "runfolder", "subd.dat"))
    g["subd_shipped"] = rows(os.path.join(ref, "subd.dat"))
    g["rhomean"] = rows(os.path.join(ref, "rhomean.dat"), 1)
    log = open(os.path.join(ref, "output"), "rb").read().decode("latin1").splitlines()

    def logged(name):
        for line in log:
            key, _, val = line.partition("=")
            if key.strip() == name:
                return float(val.strip().rstrip(",").replace("D", "E"))
        raise KeyError(name)

    g["dt_run"] = {
        "dtin": logged("DTIN"), "xlen": logged("XLEN"), "zlen": logged("ZLEN"), "brunt": logged("BRUNT"),
        # the run's namelist as its log prints it (&PARAMS, &MFLAGS)
        "params": {k.lower(): logged(k) for k in ("YLEN", "XNU", "XKAPPA", "GRAV", "RHO0", "UMAX", "XACRIT", "XBCRIT",
                                                "ZCEN", "AMP", "P", "PF", "FACKC", "FACDIR", "FACNEUMN", "FACROBIN",
                                                "NAVGINTRFC", "ISPECFILTERNL", "ISPECFILTEREXP", "NSPECFILTEREXP",
                                                "NSTEPS")},
        "grid": [int(x) for x in [l for l in log if "Number of grid points in x and z" in l][0].split(":")[1].split()],
        "nsubd": int([l for l in log if "Number of subdomains" in l][0].split()[-1]),
        "omega": [float(l.split()[-1]) for l in log if "Wave Frequency omega" in l][0],
        "cflz": [float(l.split()[-1]) for l in log if "At max CFLZ dz=" in l],
        "changes": rows(os.path.join(ref, "dtchange.dat")),
        "anim_dumps": [[int(l.split("vortanimout_")[1].split(".dat")[0]), float(l.split()[-1])]
                       for l in log if "Dumping out animation" in l],
        # the run's lines of animdump.log (the file holds other runs' lines before them)
        "animdump_log": open(os.path.join(ref, "animdump.log")).read().split("\n")[32:360],
    }
    g["_source"] = "jmsegret/IWrepo mode1_bbl run artefacts; see make_golden.py"
    with open(os.path.join(here, "reference_runs.json"), "w") as f:
        json.dump(g, f, indent=0)
    print("wrote", os.path.join(here, "reference_runs.json"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference mode1_bbl directory>")
    main(sys.argv[1])
