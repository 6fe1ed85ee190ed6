"""Drop-in for the reference's CSU.py: `python3 CSU.py ./caseFolder/`.

Builds the native solver if needed, runs it on the case folder (same input.dat, mesh.su2, restart.csv and the
same output files, solved on the GPU), then runs the case's own analysis script when it exists and its
plotting dependencies are installed (matplotlib is optional).
"""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))

if __name__ == "__main__":
    if len(sys.argv) < 2:
        print("Insert the input file")
        sys.exit(0)
    path = sys.argv[1]
    if not path.endswith("/"):
        path += "/"
    print("\nCSU - A CFD code for unstructured meshs (B200 engine):\n")
    sys.path.insert(0, ROOT)
    from csu_b200 import build
    build.build()
    rc = subprocess.call([build.EXE, path])
    if rc != 0:
        sys.exit(rc)
    script = os.path.join(path, "analisys.py")
    if os.path.exists(script):
        try:
            import matplotlib  # noqa: F401
            subprocess.call([sys.executable, script, path])
        except ImportError:
            print("matplotlib is not installed: skipping %s" % script)
