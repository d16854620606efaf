"""Generates tests/golden/obj_room.npz from the REFERENCE's own ObjSceneLoader.

Run in a tree where the reference is present (oracle/_ref/libref_oracle.so is built from its sources, with its
vendored tinyobjloader): ``python tests/golden/make_obj_golden.py``. The input is the hand-written fixture scene
tests/golden/obj/room.{meta,obj,mtl} (+ extra.mtl); the output holds everything ObjSceneLoader::Load
(src/io/scene/obj_scene_loader.cc:20-205) puts in the Scene: triangle positions, vertex normals and their flag,
geometric normals, material ids, materials, area lights, camera and point lights, as float32 bit patterns.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402


def main():
    O.build()
    r = O.RefOracle().obj_scene(os.path.join(HERE, "obj"), "room")
    assert r is not None, "the reference loader failed on the fixture"
    r = dict(r)
    r["material_names"] = np.array(r["material_names"])
    np.savez_compressed(os.path.join(HERE, "obj_room.npz"), **r)
    print(f"obj_room.npz: {len(r['positions'])} triangles, {len(r['material_names'])} materials, "
          f"{len(r['area_light_triangles'])} area lights")


if __name__ == "__main__":
    main()
