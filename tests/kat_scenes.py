"""Scenes of the reference's known-answer tests, restated with SceneBuilder.

* ``metal_scene()``: reference tests/test_metal.cpp:29-41 - back wall, floor,
  an emissive (6,6,6) quad, a metal quad, smooth (rough .02) and rough (.3)
  glass quads of IOR 1.5, and a 2x2 texture on every non-emissive triangle.
* ``fullscreen_emitter(x)``: test_metal.cpp:49, :72 - a 40x40 quad at z=3
  emitting (1,0,0), shifted by x.
* ``alpha_pair(opacity)`` and ``alpha_layers()``: tests/test_alpha.cpp:5-8,
  :13-15, :23-25.
"""
import numpy as np

from raymotion_b200.scene import Camera, RenderConfig, SceneBuilder, Texture


def _norm(v):
    v = np.asarray(v, np.float64)
    l = np.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    return v / l


def _triangle(sb, a, b, c, color, emission=(0, 0, 0), metal=0.0, ior=1.0, rough=0.5, uv=None, texture=-1):
    a, b, c = (np.asarray(p, np.float64) for p in (a, b, c))
    n = _norm(np.cross(b - a, c - a))
    sb.add_triangles([a], [b], [c], [n], [n], [n], albedo=color, emission=emission, metallic=metal, ior=ior,
                     rough=rough, uv=uv, texture=texture)


def _quad(sb, a, b, c, d, color, emission=(0, 0, 0), metal=0.0, ior=1.0, rough=0.5, texture=-1):
    tex_uv = (-.2, .1, 1.4, .2, .3, 1.7)
    uv = tex_uv if texture >= 0 else None
    _triangle(sb, a, b, c, color, emission, metal, ior, rough, uv, texture)
    _triangle(sb, a, c, d, color, emission, metal, ior, rough, uv, texture)


def metal_config():
    cfg = RenderConfig(width=96, height=64, spp=512, adapt_min=0)
    cam = Camera()
    cam.focal = cfg.width * .8660254
    cam.update_trig()
    return cam, cfg


def metal_scene(texture=True):
    sb = SceneBuilder()
    t = sb.add_texture(Texture(2, 2, np.array([[1, .1, .1], [.1, 1, .1], [.1, .1, 1], [.5, .5, .5]]))) \
        if texture else -1
    _quad(sb, (-4, -2, 7), (-4, 3, 7), (4, 3, 7), (4, -2, 7), (.7, .7, .7), texture=t)
    _quad(sb, (-4, -2, 1), (-4, -2, 7), (4, -2, 7), (4, -2, 1), (.7, .2, .1), texture=t)
    _quad(sb, (-1, 2, 3), (1, 2, 3), (1, 2, 5), (-1, 2, 5), (1, 1, 1), (6, 6, 6))
    _quad(sb, (-2, -1, 4), (-2, 1, 4), (-1, 1, 4), (-1, -1, 4), (.8, .7, .3), metal=1, texture=t)
    _quad(sb, (0, -1, 4), (0, 1, 4), (1, 1, 4), (1, -1, 4), (1, 1, 1), ior=1.5, rough=.02, texture=t)
    _quad(sb, (1, -1, 5), (1, 1, 5), (2, 1, 5), (2, -1, 5), (1, 1, 1), ior=1.5, rough=.3, texture=t)
    return sb


def fullscreen_emitter(x=0.0, alpha=1.0):
    sb = SceneBuilder()
    a, b, c, d = (x - 20, -20, 3), (x - 20, 20, 3), (x + 20, 20, 3), (x + 20, -20, 3)
    _quad(sb, a, b, c, d, (1, 1, 1), (1, 0, 0))
    packed = sb.pack()
    packed.tris["alpha"] = np.float32(alpha)
    return packed


def _surface(sb, z, alpha, emission):
    n = [(0, 0, -1)]
    sb.add_triangles([(-10, -10, z)], [(0, 10, z)], [(10, -10, z)], n, n, n, albedo=(0, 0, 0), emission=emission,
                     metallic=0, ior=1, rough=.5, alpha=alpha)


def alpha_pair(opacity):
    sb = SceneBuilder()
    _surface(sb, 1, opacity, (1, 0, 0))
    _surface(sb, 2, 1, (0, 1, 0))
    return sb


def alpha_layers():
    sb = SceneBuilder()
    for i in range(64):
        _surface(sb, 1 + i * .01, 0, (1, 0, 0))
    _surface(sb, 2, 1, (0, 1, 0))
    return sb
