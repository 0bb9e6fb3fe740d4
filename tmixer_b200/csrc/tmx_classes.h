// tmx_classes.h -- boundary node classes, in the order the reference's
// boundary_conditions() visits them (Tmixer.cpp:2023-9033).  Each boundary
// node belongs to exactly one class; cases of the reference whose closures
// are identical share a class (noted per entry).
#pragma once

#include "tmx_device.cuh"

namespace tmx {

enum BoundaryClass : unsigned char {
    K_EDGE_Y1_ZTOP = 0,  // Case 2 (H'D', :2030) and Case 3 (C'E', :2187): inlet y=1, z=nz
    K_EDGE_X1_ZTOP,      // Case 4 (G'H', :2343): inlet x=1, z=nz
    K_EDGE_XT_ZTOP,      // Case 6 (E'F', :2477): inlet x=inx, z=nz
    K_INLET1,            // Inlet1 (:2606): x=1 face
    K_INLET2,            // Inlet2 (:2668): x=inx face
    K_FACE_YT,           // Case 10 (GFF'G', :2731): inlet y=iny
    K_FACE_Y1,           // Case 11 (HDD'H', :2874) and Case 12 (CEE'C', :3016): inlet y=1 walls
    K_OUTLET,            // Case 13 (ABB'A', :3162): mixing y=1
    K_FACE_MX1,          // Case 14 (DAA'D', :3275): mixing x=1
    K_FACE_MXT,          // Case 15 (BCC'B', :3405): mixing x=mnx
    K_FACE_ZT,           // Case 16 (:3540) inlet z=nz; Case 17 (:3666) mixing z=nz and opening nodes
    K_FACE_Z1,           // Case 18 (:3888) inlet z=1; Case 19 (:4010) mixing z=1 and opening nodes
    K_EDGE_YT_ZT,        // Case 20 (G'F', :4238)
    K_EDGE_YT_Z1,        // Case 21 (GF, :4386)
    K_EDGE_X1_Z1,        // Case 22 (GH, :4534)
    K_EDGE_XT_Z1,        // Case 23 (FE, :4657)
    K_EDGE_X1_Y1,        // Case 24 (HH', :4780)
    K_EDGE_X1_YT,        // Case 25 (GG', :4910)
    K_EDGE_XT_Y1,        // Case 26 (EE', :5033)
    K_EDGE_XT_YT,        // Case 27 (FF', :5160)
    K_EDGE_Y1_Z1,        // Case 28 (HD, :5282) and Case 29 (CE, :5426)
    K_CORNER_1,          // corners 1..16 (:5572-7785): G' F' H' E' G F H E, A B A' B', D' C' C D
    K_CORNER_16 = K_CORNER_1 + 15,
    K_MEDGE_AB,          // mixing edges (:7786-8550)
    K_MEDGE_ApBp,
    K_MEDGE_AAp,
    K_MEDGE_BBp,
    K_MEDGE_AD,
    K_MEDGE_ApDp,
    K_MEDGE_BC,
    K_MEDGE_BpCp,
    K_JUNC_DD,           // edge DD' (:8551): inlet x=ia, y=1
    K_JUNC_CC,           // edge CC' (:8793): inlet x=ib, y=1
    K_NCLASSES
};
// the host's sort keys of the boundary lists hold a class in 7 bits
static_assert(K_NCLASSES <= 128, "class fits the list sort key");

// Inlets, outlet and wall faces (one kernel); edges and corners (the other).
__host__ __device__ constexpr bool is_face_class(int c)
{
    return c == K_INLET1 || c == K_INLET2 || c == K_FACE_YT || c == K_FACE_Y1 || c == K_OUTLET || c == K_FACE_MX1 ||
           c == K_FACE_MXT || c == K_FACE_ZT || c == K_FACE_Z1;
}

// Wall and outlet face nodes that the FP64 bulk kernel updates itself, one
// thread per node (the z = 1 and z = nz planes, the inlet box's y walls and
// the outlet row; whole rows and planes, so its warps stay convergent): their
// class, or -1.  Agrees with the host's classification for these classes; the
// boundary list of the FP64 form leaves them out.
__host__ __device__ inline int wall_class(const Geom& G, int b, int i, int j, int k)
{
    const bool zlo = k == 1, zhi = k == G.nz, zmid = !zlo && !zhi;
    if (b == 0) {
        if (i == 1 || i == G.inx) return -1;
        if (j == G.iny) return zmid ? K_FACE_YT : -1;
        if (j == 1) {
            if (i < G.ia || i > G.ib) return zmid ? K_FACE_Y1 : -1;
            if (i == G.ia || i == G.ib) return -1;
        }
        return zlo ? K_FACE_Z1 : zhi ? K_FACE_ZT : -1;
    }
    if (i == 1 || i == G.mnx) return -1;
    if (j == 1) return zmid ? K_OUTLET : -1;
    return zlo ? K_FACE_Z1 : zhi ? K_FACE_ZT : -1;
}

__host__ __device__ constexpr bool is_wall_class(int c)
{
    return c == K_FACE_YT || c == K_FACE_Y1 || c == K_OUTLET || c == K_FACE_ZT || c == K_FACE_Z1;
}

}  // namespace tmx
