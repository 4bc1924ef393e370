// areas.cuh -- PCA normals and point areas (the reference's --com_As 1 mode).
#pragma once

#include "common.cuh"
#include "octree.cuh"

namespace dwg {

// NormalEstimation with k nearest points (include/DWGProcess.h:152-200, PCL):
// the eigenvector of the smallest eigenvalue of the covariance of the k
// nearest points (self included), flipped to point towards the viewpoint.
// nb: [n x k] neighbour ids; view_dev: 3 floats on the device.
int pca_normals(const float* P, int n, const int* nb, int k, const float* view_dev, float* N, cudaStream_t s);

// igl::copyleft::cgal::point_areas (deps/libigl/include/igl/copyleft/cgal/
// point_areas.cpp:39-210): for point i and its k nearest (self first), keep
// those whose normal agrees with n_i, project them on their PCA plane,
// triangulate them (2-D Delaunay) and sum the Voronoi share of point i over
// its triangles (with the obtuse-triangle rules); 0 when fewer than 3 are
// kept or the result is not finite.
int point_areas(const float* P, int n, const int* nb, int k, const float* N, float* A, cudaStream_t s);

// seeded random unit normals (sin u cos v, sin u sin v, cos u), u and v
// uniform in [0, 2 pi) from splitmix64 of the index: the --in_normal 2
// --com_As 1 start (include/DWGProcess.h:643-657), whose generator the
// reference leaves unseeded
int random_normals(float* N, int n, cudaStream_t s);

// view_dev[0..2] = (upper + lower) / 2 of the points' bounding box, the
// viewpoint of the PCA normals (include/DWGProcess.h:182-187); box6_dev is
// scratch for the box (6 floats)
int box_centre(const float* P, int n, float* box6_dev, float* view_dev, cudaStream_t s);

}  // namespace dwg
