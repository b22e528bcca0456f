// Classification of the lattice nodes next to walls and open faces, computed once on the host.  The rules
// are those of the reference's LBMBoundaries (openmmapi/include/internal/LBMBoundaries.h:46-148), written
// for one domain: the same nodes, direction bits, kinds and faces, in node order.
#include "lbm_internal.h"
#include <algorithm>

namespace lbm {

static const int kCx[19] = {0, 1, -1, 0,  0, 0,  0, 1, -1,  1, -1, 0,  0,  0,  0, 1, -1, -1,  1};
static const int kCy[19] = {0, 0,  0, 1, -1, 0,  0, 1, -1, -1,  1, 1, -1,  1, -1, 0,  0,  0,  0};
static const int kCz[19] = {0, 0,  0, 0,  0, 1, -1, 0,  0,  0,  0, 1, -1, -1,  1, 1, -1,  1, -1};

static bool openAxis(const LbmLatticeParameters& l, int axis) {
    return l.face_boundary[2*axis] != LBM_BOUNDARY_PERIODIC;
}

void buildGeometry(const LbmLatticeParameters& l, int numSolid, const int* solid, Geometry& g) {
    long long n = (long long) l.nx*l.ny*l.nz;
    int size[3] = {l.nx, l.ny, l.nz};
    long long nx = l.nx, ny = l.ny;
    g = Geometry();
    g.solidNodes.assign(solid, solid + numSolid);
    std::sort(g.solidNodes.begin(), g.solidNodes.end());
    if (numSolid > 0) {
        g.fluid.assign(n, 1);
        for (int s : g.solidNodes)
            g.fluid[s] = 0;
    }
    bool anyOpen = openAxis(l, 0) || openAxis(l, 1) || openAxis(l, 2);
    bool bounceBack = numSolid > 0 && l.wall_scheme == LBM_WALL_BOUNCEBACK;
    bool regularized = numSolid > 0 && l.wall_scheme == LBM_WALL_REGULARIZED;
    if (!bounceBack && !regularized && !anyOpen)
        return;
    for (long long node = 0; node < n; node++) {
        if (!g.fluid.empty() && !g.fluid[node])
            continue;
        int index[3] = {(int) (node%nx), (int) ((node/nx)%ny), (int) (node/(nx*ny))};
        int links = 0, solidBits = 0, outsideBits = 0;
        for (int q = 1; q < 19; q++) {
            int c[3] = {kCx[q], kCy[q], kCz[q]};
            // Target x + c_q for the bounce-back links, source x - c_q for the unknown directions.
            int target[3], source[3];
            bool crosses = false, beyond = false;
            for (int a = 0; a < 3; a++) {
                target[a] = index[a] + c[a];
                source[a] = index[a] - c[a];
                crosses = crosses || (openAxis(l, a) && (target[a] < 0 || target[a] >= size[a]));
                if (source[a] < 0 || source[a] >= size[a])
                    beyond = beyond || openAxis(l, a);
                target[a] = (target[a] + size[a])%size[a];
                source[a] = (source[a] + size[a])%size[a];
            }
            if (bounceBack && !crosses && !g.fluid[target[0] + nx*(target[1] + ny*target[2])])
                links |= 1<<q;
            if (beyond)
                outsideBits |= 1<<q;
            else if (regularized && !g.fluid[source[0] + nx*(source[1] + ny*source[2])])
                solidBits |= 1<<q;
        }
        if (links != 0) {
            g.wallNodes.push_back((int) node);
            g.wallLinks.push_back(links);
        }
        if (solidBits == 0 && outsideBits == 0)
            continue;
        int nodeKind = KindWall, nodeFace = -1;
        if (solidBits == 0) {
            int velocityFace = -1, densityFace = -1, numDensityFaces = 0;
            for (int f = 0; f < 6; f++) {
                int a = f/2;
                if (!openAxis(l, a) || index[a] != (f%2 == 0 ? 0 : size[a]-1))
                    continue;
                int type = l.face_boundary[f];
                if ((type == LBM_BOUNDARY_VELOCITY || type == LBM_BOUNDARY_DENSITY_VELOCITY) && velocityFace < 0)
                    velocityFace = f;
                if (type == LBM_BOUNDARY_DENSITY && numDensityFaces++ == 0)
                    densityFace = f;
            }
            if (velocityFace >= 0) {
                nodeKind = (l.face_boundary[velocityFace] == LBM_BOUNDARY_DENSITY_VELOCITY ? KindDensityVelocity : KindVelocity);
                nodeFace = velocityFace;
            }
            else {
                nodeKind = (numDensityFaces == 1 ? KindDensity : KindDensityAtRest);
                nodeFace = densityFace;
            }
        }
        g.boundaryNodes.push_back((int) node);
        g.unknown.push_back(solidBits | outsideBits);
        g.solidBits.push_back(solidBits);
        g.kind.push_back(nodeKind);
        g.face.push_back(nodeFace);
    }
}

// The static part of the wall momentum of a step, -2 c_q w_q for every link from a solid node into the fluid, which
// the reference's GPU kernels keep apart from the momentum that they store per wall entry (CommonLBMKernels.cpp:
// 297-311 for bounce-back, :356-366 for the solid directions of the boundary nodes; added back at :1932 and :1938).  A bounce-back link is stored
// here from its fluid side (bit q of x where x + c_q is solid), so the link from the solid node has velocity -c_q.
void staticWallMomentum(const LbmLatticeParameters& l, const Geometry& g, double momentum[3]) {
    momentum[0] = momentum[1] = momentum[2] = 0;
    auto weight = [](int q) { return q == 0 ? 1.0/3.0 : q < 7 ? 1.0/18.0 : 1.0/36.0; };
    if (l.wall_scheme == LBM_WALL_BOUNCEBACK)
        for (size_t i = 0; i < g.wallNodes.size(); i++)
            for (int q = 1; q < 19; q++)
                if (g.wallLinks[i] & (1<<q)) {
                    momentum[0] += 2.0*kCx[q]*weight(q);
                    momentum[1] += 2.0*kCy[q]*weight(q);
                    momentum[2] += 2.0*kCz[q]*weight(q);
                }
    for (size_t b = 0; b < g.boundaryNodes.size(); b++)
        for (int q = 1; q < 19; q++)
            if (g.solidBits[b] & (1<<q)) {
                momentum[0] -= 2.0*kCx[q]*weight(q);
                momentum[1] -= 2.0*kCy[q]*weight(q);
                momentum[2] -= 2.0*kCz[q]*weight(q);
            }
}

} // namespace lbm
