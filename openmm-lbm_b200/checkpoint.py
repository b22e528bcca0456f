"""The reference's checkpoint formats around the kernel's stream.

- LBMForce.createCheckpoint(context) (LBMForceImpl::createCheckpoint, openmmapi/src/LBMForceImpl.cpp:568-573) writes
  a header (LBMForceImpl::writeCheckpointHeader, :514-528) before the kernel's stream: the tag "LBMCKPT1", the
  version 6, the platform's name after its int length, and 14 ints: nx, ny, nz, the number of coupled particles, the
  drag scheme, the fluid fluctuations, the wall scheme, the boundary types of the six faces and the interpolation
  stencil.  readCheckpointHeader (:530-566) also reads versions 1 to 5, which hold fewer of the ints (version + 3 for
  versions 1 to 4, 13 for version 5), with the defaults of the settings that did not exist yet.
- openmmlbm.saveCheckpoint() with one domain (python/openmmlbm.i:513-550, LBMForceImpl.cpp:580-598) writes a file: the
  tag "OPENMMLBM-CHECKPOINT-1\\n", the int64 lengths of the OpenMM checkpoint and of the force checkpoint, and the two.

All integers are little-endian, as the reference writes them on x86-64 and aarch64.
"""
import struct

from .abi import LbmError, LBM_ERR_CHECKPOINT

CHECKPOINT_TAG = b'LBMCKPT1'
CHECKPOINT_VERSION = 6
FILE_TAG = b'OPENMMLBM-CHECKPOINT-1\n'
# LBMForce enumerations (openmmapi/include/LBMForce.h:61-138): Explicit, BounceBack, Periodic, NearestNode.
_DEFAULT_HEADER = [0, 0, 0, 0, 0, 0, 0] + [0]*6 + [0]


def _fail(message):
    raise LbmError(LBM_ERR_CHECKPOINT, message)


def header_values(lattice, num_particles):
    """The 14 ints of the header for a lattice (LbmLatticeParameters) with num_particles coupled particles."""
    return ([lattice.nx, lattice.ny, lattice.nz, num_particles, lattice.drag_scheme,
             1 if lattice.fluid_fluctuations else 0, lattice.wall_scheme] +
            [lattice.face_boundary[f] for f in range(6)] + [lattice.interpolation_stencil])


def write_header(platform, lattice, num_particles, version=CHECKPOINT_VERSION):
    """The header of LBMForce.createCheckpoint() (version 6; older versions for tests of the reader)."""
    name = platform.encode()
    values = header_values(lattice, num_particles)[:_header_length(version)]
    return (CHECKPOINT_TAG + struct.pack('<ii', version, len(name)) + name +
            struct.pack('<%di' % len(values), *values))


def _header_length(version):
    return version + 3 if version <= 4 else 13 if version == 5 else 14


def read_header(data, platform, lattice, num_particles):
    """Check the header of a force checkpoint against the platform's name and the lattice of the Context, as
    readCheckpointHeader does, with its messages; returns the offset of the kernel's stream."""
    data = bytes(data)
    if data[:8] != CHECKPOINT_TAG:
        _fail('LBMForce: the data are not a checkpoint written by LBMForce::createCheckpoint()')
    if len(data) < 12:
        _fail('LBMForce: unsupported checkpoint version')
    version, = struct.unpack_from('<i', data, 8)
    if version < 1 or version > CHECKPOINT_VERSION:
        _fail('LBMForce: unsupported checkpoint version')
    if len(data) < 16:
        _fail('LBMForce: the checkpoint is damaged')
    length, = struct.unpack_from('<i', data, 12)
    if length < 0 or length > 1000 or len(data) < 16 + length:
        _fail('LBMForce: the checkpoint is damaged')
    written = data[16:16 + length].decode(errors='replace')
    if written != platform:
        _fail('LBMForce: the checkpoint was written on the platform %s, not on %s' % (written, platform))
    count = _header_length(version)
    start = 16 + length
    if len(data) < start + 4*count:
        _fail('LBMForce: the checkpoint was written for a different grid size or number of coupled particles')
    header = list(_DEFAULT_HEADER)
    header[:count] = struct.unpack_from('<%di' % count, data, start)
    expected = header_values(lattice, num_particles)
    if header[:4] != expected[:4]:
        _fail('LBMForce: the checkpoint was written for a different grid size or number of coupled particles')
    if header[4] != expected[4]:
        _fail('LBMForce: the checkpoint was written with a different drag scheme')
    if header[5] != expected[5]:
        _fail('LBMForce: the checkpoint was written %s fluid fluctuations, and this Context has them %s' %
              ('with' if header[5] else 'without', 'on' if expected[5] else 'off'))
    if header[6] != expected[6]:
        _fail('LBMForce: the checkpoint was written with a different wall scheme')
    if header[7:13] != expected[7:13]:
        _fail('LBMForce: the checkpoint was written with different boundary types of the faces (setFaceBoundary())')
    if header[13] != expected[13]:
        _fail('LBMForce: the checkpoint was written with a different interpolation stencil')
    return start + 4*count


def pack_file(openmm_data, force_data):
    """The file of saveCheckpoint() with one domain."""
    return FILE_TAG + struct.pack('<qq', len(openmm_data), len(force_data)) + openmm_data + force_data


def unpack_file(data, name='the file'):
    """(OpenMM checkpoint, force checkpoint) of a file written by saveCheckpoint() with one domain."""
    if not data.startswith(FILE_TAG):
        raise ValueError('%s is not a checkpoint written by openmmlbm.saveCheckpoint()' % name)
    start = len(FILE_TAG) + 16
    if len(data) < start:
        raise ValueError('%s is truncated or damaged' % name)
    openmm_length, force_length = struct.unpack_from('<qq', data, len(FILE_TAG))
    if openmm_length < 0 or force_length < 0 or len(data) != start + openmm_length + force_length:
        raise ValueError('%s is truncated or damaged' % name)
    return data[start:start + openmm_length], data[start + openmm_length:]
