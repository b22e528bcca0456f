"""TEST INFRASTRUCTURE: the kernel stream of the reference's GPU platforms, restated for one domain, to read the
checkpoints of the B200 kernel and to build the streams that the reference's CUDA kernel writes.

CommonCalcLBMForceKernel::createCheckpoint / loadCheckpoint (platforms/common/src/CommonLBMKernels.cpp:2019-2058):
int element size E (8 in double and mixed precision, 4 in single, :243-244); int flags[2] = {noiseDrawn,
hasAdvanced}; then each array that exists, as it is on the device:
    populations          19*N values of E bytes, f_q - w_q, [q*N + node]                       (:251, :1961-1966)
    noise                P float4 (N(0,1) numbers drawn for the next step), when P > 0          (:723)
    particleWallMomentum 3*P values of E bytes, [a*P + i], when P > 0                          (:666)
    wallExchange         3*max(1, S) values of E bytes, [a*S + entry]; one entry per solid node  (:296-331, :401)
    boundaryExchange     3*B values of E bytes, [a*B + b], when B > 0 boundary nodes           (:368-379)
getWallForce() (:1918-1945) reports, when there are solid nodes and the fluid has advanced, the sum of the entries of
the last three arrays plus the static parts: -2 c_q w_q for every link from a solid node into the fluid that crosses
no open face, with bounce-back (:297-311), and for every solid direction of a boundary node (:356-366).

Only tests use this module.
"""
import struct

import numpy as np

# D3Q19 in the reference's order (openmmapi/include/internal/D3Q19.h:29-31).
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1])
W = np.array([1/3] + [1/18]*6 + [1/36]*12)


def _dtype(element_size):
    if element_size not in (4, 8):
        raise ValueError('element size %d' % element_size)
    return np.dtype('<f8') if element_size == 8 else np.dtype('<f4')


def stream_bytes(element_size, num_nodes, num_particles, num_solid, num_boundary):
    e = element_size
    size = 12 + 19*num_nodes*e
    if num_particles > 0:
        size += 16*num_particles + 3*num_particles*e
    size += 3*max(1, num_solid)*e
    if num_boundary > 0:
        size += 3*num_boundary*e
    return size


def read_stream(data, num_nodes, num_particles, num_solid, num_boundary):
    """The arrays of a stream, as loadCheckpoint reads them; 'end' is the offset after the last array."""
    e, noise_drawn, has_advanced = struct.unpack_from('<iii', data, 0)
    t = _dtype(e)
    offset = 12

    def take(count, dtype):
        nonlocal offset
        values = np.frombuffer(data, dtype=dtype, count=count, offset=offset).astype(np.float64)
        offset += count*dtype.itemsize
        return values

    out = {'element_size': e, 'noise_drawn': noise_drawn, 'has_advanced': has_advanced,
           'populations': take(19*num_nodes, t)}
    if num_particles > 0:
        out['noise'] = take(4*num_particles, np.dtype('<f4')).reshape(num_particles, 4)
        out['particle_wall'] = take(3*num_particles, t).reshape(3, num_particles)
    out['wall'] = take(3*max(1, num_solid), t).reshape(3, max(1, num_solid))
    if num_boundary > 0:
        out['boundary'] = take(3*num_boundary, t).reshape(3, num_boundary)
    out['end'] = offset
    return out


def stored_wall_momentum(arrays, num_solid):
    """The sum of the stored wall entries (getWallForce without the static parts), lattice units."""
    if num_solid == 0 or not arrays['has_advanced']:
        return np.zeros(3)
    total = arrays['wall'].sum(axis=1)
    if 'boundary' in arrays:
        total = total + arrays['boundary'].sum(axis=1)
    if 'particle_wall' in arrays:
        total = total + arrays['particle_wall'].sum(axis=1)
    return total


def write_stream(element_size, populations, has_advanced, wall_entries, num_particles, num_solid, num_boundary,
                 particle_wall=None, boundary=None, noise=None):
    """A stream as createCheckpoint writes it.  wall_entries: (3, max(1, S)); particle_wall: (3, P); boundary:
    (3, B); noise: (P, 4) numbers drawn for the next step (noiseDrawn = 1), or None (zeros, noiseDrawn = 0)."""
    t = _dtype(element_size)
    parts = [struct.pack('<iii', element_size, 0 if noise is None else 1, 1 if has_advanced else 0),
             np.asarray(populations, dtype=np.float64).astype(t).tobytes()]
    if num_particles > 0:
        n = np.zeros((num_particles, 4)) if noise is None else np.asarray(noise)
        parts.append(n.astype('<f4').tobytes())
        pw = np.zeros((3, num_particles)) if particle_wall is None else np.asarray(particle_wall)
        parts.append(pw.astype(t).tobytes())
    parts.append(np.asarray(wall_entries, dtype=np.float64).reshape(3, max(1, num_solid)).astype(t).tobytes())
    if num_boundary > 0:
        b = np.zeros((3, num_boundary)) if boundary is None else np.asarray(boundary)
        parts.append(b.astype(t).tobytes())
    return b''.join(parts)


def static_wall_momentum(lattice, solid_nodes, boundary_solid_bits):
    """The static parts of the wall momentum (lattice units) for a lattice (LbmLatticeParameters), its solid nodes
    and the solid direction bits of its boundary nodes (oracle.find_boundaries()[2])."""
    nx, ny, nz = lattice.nx, lattice.ny, lattice.nz
    size = (nx, ny, nz)
    is_open = [lattice.face_boundary[2*a] != 0 for a in range(3)]
    fluid = np.ones(nx*ny*nz, dtype=bool)
    fluid[np.asarray(solid_nodes, dtype=np.int64)] = False
    momentum = np.zeros(3)
    if lattice.wall_scheme == 0:
        for node in solid_nodes:
            index = (node % nx, (node//nx) % ny, node//(nx*ny))
            for q in range(1, 19):
                c = (CX[q], CY[q], CZ[q])
                target = [index[a] + c[a] for a in range(3)]
                if any(is_open[a] and not 0 <= target[a] < size[a] for a in range(3)):
                    continue
                target = [target[a] % size[a] for a in range(3)]
                if fluid[target[0] + nx*(target[1] + ny*target[2])]:
                    momentum -= 2.0*W[q]*np.array(c, dtype=float)
    for bits in boundary_solid_bits:
        for q in range(1, 19):
            if int(bits) & (1 << q):
                momentum -= 2.0*W[q]*np.array([CX[q], CY[q], CZ[q]], dtype=float)
    return momentum
