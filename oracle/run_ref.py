"""Run a reference SMAUG binary built by oracle/build_ref.py (test infrastructure).

The binary reads its compile-time CFGFILE ("ref.ini") from the working
directory and writes out/ref_<it>.out every step (PCFGSAVEFREQUENCY 1):
file _k holds the state after k steps, its header time is one step ahead
(src/iosmaug.c:509-523,1129-1132).  Per-step wall times come from the
reference's own "time total=" line (src/iosmaug.c:1127).

Usage (on the GPU box):
  python oracle/run_ref.py BINARY INI RUNDIR [KEEP_STEPS comma list]
"""
import os
import re
import shutil
import subprocess
import sys


def run(binary, ini, rundir, keep=None, timeout=3000):
    os.makedirs(os.path.join(rundir, "out"), exist_ok=True)
    shutil.copy(ini, os.path.join(rundir, "ref.ini"))
    with open(os.path.join(rundir, "stdout.txt"), "w") as log:
        rc = subprocess.call([os.path.abspath(binary)], cwd=rundir, stdout=log,
                             stderr=subprocess.STDOUT, timeout=timeout)
    times = []
    with open(os.path.join(rundir, "stdout.txt")) as f:
        for line in f:
            m = re.search(r"^step (\d+) .* time total=([0-9.eE+-]+)", line)
            if m:
                times.append((int(m.group(1)), float(m.group(2))))
    if keep is not None:
        for fn in os.listdir(os.path.join(rundir, "out")):
            m = re.match(r"ref_(\d+)\.out$", fn)
            if m and int(m.group(1)) not in keep:
                os.remove(os.path.join(rundir, "out", fn))
    with open(os.path.join(rundir, "times.txt"), "w") as f:
        for s, t in times:
            f.write("%d %.6f\n" % (s, t))
    # keep only the tail of the (verbose) stdout
    with open(os.path.join(rundir, "stdout.txt")) as f:
        lines = f.readlines()
    with open(os.path.join(rundir, "stdout_tail.txt"), "w") as f:
        f.writelines(lines[-200:])
    os.remove(os.path.join(rundir, "stdout.txt"))
    return rc, times


if __name__ == "__main__":
    a = sys.argv[1:]
    keep = None
    if len(a) > 3:
        keep = set(int(x) for x in a[3].split(","))
    rc, times = run(a[0], a[1], a[2], keep)
    print("rc", rc, "steps", len(times))
    sys.exit(rc)
