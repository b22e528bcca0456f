"""CPU tests of the reference's checkpoint formats around the kernel's stream (lbm_b200.checkpoint): the header of
LBMForce.createCheckpoint() (LBMForceImpl::writeCheckpointHeader / readCheckpointHeader, openmmapi/src/
LBMForceImpl.cpp:514-566) with the versions 1 to 6 that the reference reads and its messages, the file of
saveCheckpoint() with one domain (python/openmmlbm.i:513-586), and the oracle's restatement of the GPU platforms'
kernel stream (CommonLBMKernels.cpp:2019-2058) that the GPU tests read the B200 kernel's checkpoints with."""
import struct

import numpy as np
import pytest

from lbm_b200 import LBMForce, checkpoint
from lbm_b200.abi import LbmError

import checkpoint_format


def lattice(**fields):
    """The lattice of a 6x5x4 force, with fields of LbmLatticeParameters set directly (face_boundary: {face: type})."""
    force = LBMForce()
    force.setGridSize(6, 5, 4)
    lat = force.latticeParameters(np.array([3.0, 2.5, 2.0]), 0.01, np.ones(3))
    for name, value in fields.items():
        if name == 'face_boundary':
            for face, kind in value.items():
                lat.face_boundary[face] = kind
        else:
            setattr(lat, name, value)
    return lat


def test_header_bytes():
    lat = lattice(drag_scheme=LBMForce.Centered, interpolation_stencil=LBMForce.Keys, wall_scheme=LBMForce.Regularized,
                  face_boundary={LBMForce.YMax: LBMForce.Density})
    data = checkpoint.write_header('CUDA', lat, 3)
    expected = (b'LBMCKPT1' + struct.pack('<ii', 6, 4) + b'CUDA' +
                struct.pack('<14i', 6, 5, 4, 3, 1, 0, 1, 0, 0, 0, 2, 0, 0, 3))
    assert data == expected
    assert checkpoint.read_header(data + b'stream', 'CUDA', lat, 3) == len(expected)


@pytest.mark.parametrize('version,count', [(1, 4), (2, 5), (3, 6), (4, 7), (5, 13), (6, 14)])
def test_old_header_versions_take_the_defaults(version, count):
    """Versions 1 to 5 hold fewer ints; the settings that did not exist yet take the values of that time: the
    explicit drag (1), no fluctuations (2), bounce-back (3), periodic faces (4), the nearest node (5)."""
    plain = lattice()
    data = checkpoint.write_header('CUDA', plain, 0, version=version)
    assert len(data) == 8 + 8 + 4 + 4*count
    assert checkpoint.read_header(data, 'CUDA', plain, 0) == len(data)
    newer = [('drag_scheme', LBMForce.Centered, 'drag scheme', 2), ('fluid_fluctuations', 1, 'fluctuations', 3),
             ('wall_scheme', LBMForce.Regularized, 'wall scheme', 4),
             ('face_boundary', {LBMForce.XMin: LBMForce.Velocity}, 'boundary types', 5),
             ('interpolation_stencil', LBMForce.Trilinear, 'interpolation stencil', 6)]
    for name, value, message, first in newer:
        lat = lattice(**{name: value})
        if version < first:
            # The checkpoint predates the setting, so it was written with its default.
            with pytest.raises(LbmError, match=message):
                checkpoint.read_header(checkpoint.write_header('CUDA', lat, 0, version=version), 'CUDA', lat, 0)
        else:
            assert checkpoint.read_header(checkpoint.write_header('CUDA', lat, 0, version=version), 'CUDA', lat, 0)


def test_header_errors():
    lat = lattice()
    data = checkpoint.write_header('CUDA', lat, 2)
    cases = [(b'LBMCKPT2' + data[8:], 'not a checkpoint written by LBMForce::createCheckpoint'),
             (data[:8] + struct.pack('<i', 7) + data[12:], 'unsupported checkpoint version'),
             (data[:8] + struct.pack('<i', 0) + data[12:], 'unsupported checkpoint version'),
             (data[:12] + struct.pack('<i', 1001) + data[16:], 'the checkpoint is damaged'),
             (data[:30], 'different grid size or number of coupled particles')]
    for bad, message in cases:
        with pytest.raises(LbmError, match=message):
            checkpoint.read_header(bad, 'CUDA', lat, 2)
    with pytest.raises(LbmError, match='written on the platform CUDA, not on Reference'):
        checkpoint.read_header(data, 'Reference', lat, 2)
    with pytest.raises(LbmError, match='different grid size or number of coupled particles'):
        checkpoint.read_header(data, 'CUDA', lat, 3)
    fluct = lattice(fluid_fluctuations=1)
    with pytest.raises(LbmError, match='written without fluid fluctuations, and this Context has them on'):
        checkpoint.read_header(data, 'CUDA', fluct, 2)


def test_checkpoint_file():
    data = checkpoint.pack_file(b'openmm', b'force-data')
    assert data == b'OPENMMLBM-CHECKPOINT-1\n' + struct.pack('<qq', 6, 10) + b'openmm' + b'force-data'
    assert checkpoint.unpack_file(data) == (b'openmm', b'force-data')
    with pytest.raises(ValueError, match='truncated or damaged'):
        checkpoint.unpack_file(data[:-1])
    with pytest.raises(ValueError, match='not a checkpoint written by openmmlbm.saveCheckpoint'):
        checkpoint.unpack_file(b'OPENMMLBM-CHECKPOINT-2\n' + data[23:])


@pytest.mark.parametrize('element_size', [4, 8])
def test_stream_restatement_round_trip(element_size):
    rng = np.random.default_rng(5)
    n, p, s, b = 120, 3, 7, 11
    populations = rng.normal(size=19*n)*1e-2
    wall = rng.normal(size=(3, s))
    boundary = rng.normal(size=(3, b))
    particle_wall = rng.normal(size=(3, p))
    noise = rng.normal(size=(p, 4))
    data = checkpoint_format.write_stream(element_size, populations, True, wall, p, s, b, particle_wall, boundary,
                                          noise)
    assert len(data) == checkpoint_format.stream_bytes(element_size, n, p, s, b)
    arrays = checkpoint_format.read_stream(data, n, p, s, b)
    assert arrays['end'] == len(data)
    assert (arrays['element_size'], arrays['noise_drawn'], arrays['has_advanced']) == (element_size, 1, 1)
    cast = np.float64 if element_size == 8 else np.float32
    assert (arrays['populations'] == populations.astype(cast)).all()
    assert (arrays['noise'] == noise.astype(np.float32)).all()
    stored = [a.astype(cast).astype(np.float64) for a in (wall, boundary, particle_wall)]
    total = stored[0].sum(axis=1) + stored[1].sum(axis=1) + stored[2].sum(axis=1)
    assert np.allclose(checkpoint_format.stored_wall_momentum(arrays, s), total, rtol=1e-12, atol=0)


def test_static_wall_momentum_of_a_plane():
    """Bounce-back at the plane j = 0 of a periodic 6x5x4 lattice: every solid node has 5 links into the fluid above
    (c_y = +1) and 5 below (c_y = -1, through the periodic boundary), so the static momentum cancels; with the face
    y = 0 open only the links upwards count: 24 nodes x (-2 (1/18 + 4/36)) along y."""
    solid = [i + 30*k for k in range(4) for i in range(6)]
    m = checkpoint_format.static_wall_momentum(lattice(), solid, [])
    assert np.allclose(m, 0, atol=1e-14)
    lat = lattice(face_boundary={LBMForce.YMin: LBMForce.Velocity, LBMForce.YMax: LBMForce.Velocity})
    m = checkpoint_format.static_wall_momentum(lat, solid, [])
    assert np.allclose(m, [0, -24*2*(1/18 + 4/36), 0], rtol=1e-14, atol=1e-14)
