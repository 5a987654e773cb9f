// Host-side convex polyhedron construction (see hull.cpp).
#pragma once
#include <string>
#include <vector>

namespace b3hull {

struct Face {
    float plane[4];
    std::vector<int> indices;
};

struct Polyhedron {
    std::vector<float> vertices;     // xyz triples (hull vertices, input order)
    std::vector<Face> faces;
    std::vector<float> uniqueEdges;  // xyz triples
    float localCenter[3] = {0, 0, 0};
    float aabbMin[3] = {0, 0, 0}, aabbMax[3] = {0, 0, 0};
    float mC[3] = {0, 0, 0}, mE[3] = {0, 0, 0};
    // distance from localCenter to the nearest facet of the exact hull
    // (before the coplanar weld): the hull's support about its local centre
    // is at least this in every direction
    double inradius = 0.0;
};

bool compute_polyhedron(const float* pts, int n, Polyhedron& out, std::string* err);

}  // namespace b3hull
