"""Materializes test cases as short case folders (the reference builds paths in char[50] buffers)."""
import gzip
import hashlib
import os

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
CASES = sorted(d for d in os.listdir(os.path.join(GOLDEN, "cases"))) if os.path.isdir(
    os.path.join(GOLDEN, "cases")) else []

# Settings the engine runs the reference cases with in the golden vectors: the restart cases start from
# the free stream, and the LU-SGS wedge uses DPLUR (LU-SGS is checked separately, at convergence).
GOLDEN_OVERRIDES = {
    "caseBL": {"restart": "0"},
    "caseBL_turb": {"restart": "0"},
    "caseNACA0012": {"restart": "0"},
    "caseWedge": {"timeScheme": "DPLUR", "Nlinear": "4", "CFL": "10.0"},
}

INVISCID = ["caseChannel", "caseCylinder", "caseCylinderAxi", "caseDiamond", "caseSod", "caseSodRef",
            "caseWedge", "caseWedgeAxi", "caseWedgeQuad"]


def read_input(name):
    with open(os.path.join(GOLDEN, "cases", name, "input.dat")) as f:
        return f.read()


def read_mesh(name):
    with gzip.open(os.path.join(GOLDEN, "cases", name, "mesh.su2.gz"), "rt") as f:
        return f.read()


def override(text, kv):
    """Replace or append `name, value` lines of an input.dat text."""
    lines = text.split("\n")
    done = set()
    for i, line in enumerate(lines):
        key = line.split(",")[0].strip() if "," in line else None
        if key in kv:
            lines[i] = "%s, %s" % (key, kv[key])
            done.add(key)
    extra = ["%s, %s" % (k, v) for k, v in kv.items() if k not in done]
    body = "\n".join(lines).rstrip("\n")
    return body + "\n" + "".join(e + "\n" for e in extra)


def write_case(text, mesh, tag=""):
    h = hashlib.sha1((text + tag).encode() + mesh[:4096].encode() + str(len(mesh)).encode()).hexdigest()[:10]
    wd = "/tmp/cs%s/" % h
    os.makedirs(wd, exist_ok=True)
    with open(wd + "input.dat", "w") as f:
        f.write(text)
    p = wd + "mesh.su2"
    if not os.path.exists(p) or os.path.getsize(p) != len(mesh):
        with open(p, "w") as f:
            f.write(mesh)
    return wd


def materialize(name, kv=None):
    text = read_input(name)
    if kv:
        text = override(text, kv)
    return write_case(text, read_mesh(name), name)


def is_tube(wd):
    with open(wd + "input.dat") as f:
        for line in f:
            if line.replace(" ", "").startswith("tube,"):
                return line.split(",")[1].strip() == "1"
    return False
