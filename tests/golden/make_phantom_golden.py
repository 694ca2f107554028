"""Generates tests/golden/forbild_phantoms.npz: the FORBILD-style head and
jaw phantoms of the reference (emil_code/phantoms/head_phantom.py
build_head_phantom, jaw_phantom.py build_jaw_phantom) flattened to their
shapes, so the tests can voxelise and project them without the reference.

The builders are the reference's own code, run here against this
repository's tomo3D object layer (ct-2_b200/tomo3D.py, imported as the
`tomo3D` they import); only Python-2 syntax is rewritten (print statements,
tabs).  Each leaf shape is recorded as data:

* ellipsoids: (x0, y0, z0, att, ax, ay, az, alpha, beta);
* gen_objects: att, the counts (nsurf, nplane, nellipsoid, ncyl, ncone) and
  the surface table (twelve frame rows, semi-axis arrays) exactly as
  gen_object.table() hands it to gen_shape_proj / gen_obj_embed.

It reads the reference's sources at generation time only.

Run: python tests/golden/make_phantom_golden.py <reference root>
     (or set CT2_REFERENCE_ROOT)
"""
import os
import re
import sys
import types

import numpy as np

from refroot import reference_root  # noqa: E402

REF = os.path.join(reference_root(), "emil_code", "phantoms")
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "forbild_phantoms.npz")
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "ct-2_b200"))


def load(name):
    src = open(os.path.join(REF, name + ".py")).read().expandtabs(8)
    src = re.sub(r"^(\s*)print (.*)$", r"\1print(\2)", src, flags=re.M)
    mod = types.ModuleType(name)
    mod.__dict__["__name__"] = name  # not __main__: the demo block stays off
    exec(compile(src, name + ".py", "exec"), mod.__dict__)
    return mod


def leaves(ph):
    for c in ph.components:
        if hasattr(c, "components"):
            yield from leaves(c)
        else:
            yield c


def flatten(ph, tag, out):
    import tomo3D as T
    ell, gatt, counts, frames, axes = [], [], [], [], []
    for c in leaves(ph):
        if isinstance(c, T.ellipsoid):
            ell.append([c.x0, c.y0, c.z0, c.att, c.ax, c.ay, c.az, c.alpha, c.beta])
        elif isinstance(c, T.gen_object):
            tab = c.table()
            gatt.append(c.att)
            counts.append([tab[0], tab[13], tab[14], tab[18], tab[21]])
            frames.append(np.stack(tab[1:13]).astype(np.float32))
            axes.append(np.concatenate([np.asarray(a, np.float32) for a in
                                        tab[15:18] + tab[19:21] + tab[22:24]]))
        else:
            raise TypeError("unexpected shape %r" % (c,))
    out[tag + "_ell"] = np.array(ell, np.float64).reshape(-1, 9)
    out[tag + "_gatt"] = np.array(gatt, np.float64)
    out[tag + "_counts"] = np.array(counts, np.int32).reshape(-1, 5)
    out[tag + "_frames"] = np.concatenate(frames, axis=1) if frames else np.zeros((12, 0),
                                                                                 np.float32)
    out[tag + "_axes"] = np.concatenate(axes) if axes else np.zeros(0, np.float32)
    print(tag, len(ell), "ellipsoids,", len(gatt), "surface objects")


def main():
    out = {}
    flatten(load("head_phantom").build_head_phantom(), "head", out)
    flatten(load("jaw_phantom").build_jaw_phantom(), "jaw", out)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
