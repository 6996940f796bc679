"""Photon-map emitter set-up: the host side of SceneData::rebuild_caustics
(src/scene.rs:35-74) producing RtPhotonParams for rt_photon_build."""
import math

import numpy as np

import ctypes as C

from . import abi


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


def disk_emitter(sun_dir, sun_color, n_photons):
    """PhotonMap::build (photon.rs:41-94): a disk facing sun_dir sized to the scene."""
    e = abi.RtPhotonEmitter()
    e.type = abi.RT_EMIT_DISK
    e.dir = (C.c_float * 3)(*[float(x) for x in sun_dir])
    e.color = (C.c_float * 3)(*[float(x) for x in sun_color])
    e.n_photons = int(n_photons)
    return e


def quad_emitter(corner, u, v, color, n_photons):
    """PhotonMap::build_from_quad (photon.rs:97-135): cosine-weighted quad source."""
    e = abi.RtPhotonEmitter()
    e.type = abi.RT_EMIT_QUAD
    fl = lambda x: (C.c_float * 3)(*[float(y) for y in x])
    e.corner, e.u, e.v, e.color = fl(corner), fl(u), fl(v), fl(color)
    e.n_photons = int(n_photons)
    return e


def sun_emitter(n_photons):
    """The Physical sky's sun as the caustic source (scene.rs:40-52); the library
    derives the direction and colour from the scene's background."""
    e = abi.RtPhotonEmitter()
    e.type = abi.RT_EMIT_SUN
    e.n_photons = int(n_photons)
    return e


def light_emitter(light, n_photons, target=None):
    """Entry `light` of the scene's light list (a quad) as a cosine-weighted quad
    source (PhotonMap::build_from_quad, photon.rs:97-135) coloured by its
    material's emission; the library reads the quad and the colour.  target:
    (centre, radius) of a sphere around the caustic-casting objects, toward
    which every photon is sent with its power reweighted (a projection map of
    the same expected caustics; see RtPhotonEmitter.target)."""
    e = abi.RtPhotonEmitter()
    e.type = abi.RT_EMIT_LIGHT
    e.light = int(light)
    e.n_photons = int(n_photons)
    if target is not None:
        (cx, cy, cz), r = target
        e.target = (C.c_float * 4)(float(cx), float(cy), float(cz), float(r))
    return e


def light_params(builder, n_photons, gather_radius, knn_k=0, seed=0, target=None):
    """Caustic photons emitted from every quad of the light list, the total
    split evenly between them (optionally aimed at a projection sphere).  The
    reference's rebuild_caustics emits from the env disk when the scene has an
    env map (scene.rs:52-73); scenes whose caustics come from their area lights
    use this instead."""
    quads = [i for i, (kind, _) in enumerate(builder._lights) if kind == "quad"]
    if not quads:
        raise ValueError("the scene has no light quad")
    if len(quads) > abi.RT_MAX_EMITTERS:
        raise ValueError("more light quads than emitters")
    base, rem = divmod(int(n_photons), len(quads))
    ems = [light_emitter(li, base + (1 if k < rem else 0), target) for k, li in enumerate(quads)]
    return photon_params(ems, gather_radius, knn_k, seed)


def bounding_sphere(V):
    """(centre, radius) of a sphere holding the points V (n, 3): the box centre
    and the farthest point from it, padded by 1e-4 relative."""
    V = np.asarray(V, np.float64)
    c = (V.min(0) + V.max(0)) * 0.5
    r = float(np.sqrt(((V - c) ** 2).sum(1).max())) * (1.0 + 1e-4)
    return tuple(float(x) for x in c), r


def shard_params(params, world, rank):
    """The same build restricted to rank's contiguous share of the emission
    order (RtPhotonParams.first_photon / shard_photons)."""
    total = sum(params.emitters[i].n_photons for i in range(params.n_emitters))
    base, rem = divmod(total, int(world))
    first = rank * base + min(rank, rem)
    q = abi.RtPhotonParams()
    C.pointer(q)[0] = params
    q.first_photon = first
    q.shard_photons = base + (1 if rank < rem else 0)
    if q.shard_photons == 0:
        raise ValueError("a shard with no photons")
    return q


def photon_params(emitters, gather_radius, knn_k=0, seed=0):
    if not (1 <= len(emitters) <= abi.RT_MAX_EMITTERS):
        raise ValueError("1..8 emitters")
    p = abi.RtPhotonParams()
    p.n_emitters = len(emitters)
    for i, e in enumerate(emitters):
        p.emitters[i] = e
    p.gather_radius = float(gather_radius)
    p.knn_k = int(knn_k)
    p.seed = int(seed)
    return p


def caustic_params(builder, n_photons, gather_radius, knn_k=0, seed=0, env_dir=None, env_color=None):
    """rebuild_caustics emitter choice (scene.rs:40-73): a Physical sky → its sun;
    an env map → disk facing a bright env direction (computed by the caller as the reference does from 8
    CDF samples), otherwise the first [[lights]] quad with its `color`."""
    if builder.bg.get("type") == abi.RT_BG_PHYSICAL:
        return photon_params([sun_emitter(n_photons)], gather_radius, knn_k, seed)
    if env_dir is not None:
        return photon_params([disk_emitter(env_dir, env_color, n_photons)], gather_radius, knn_k, seed)
    quads = [builder.quads[i] for kind, i in builder._lights if kind == "quad"]
    if not quads:
        raise ValueError("no caustic emitter: the scene has neither an env map nor a light quad")
    q, u, v, mat = quads[0]
    color = list(builder.materials[mat].albedo)
    return photon_params([quad_emitter(q, u, v, color, n_photons)], gather_radius, knn_k, seed)
