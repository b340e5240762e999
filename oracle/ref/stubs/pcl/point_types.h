// Stand-in for pcl/point_types.h, written for compiling the reference's index kernels in place
// (oracle/ref/Makefile): the point types the reference's headers name, as plain structs.
#pragma once

namespace pcl {
struct PointXYZ { float x, y, z; };
struct Normal { float normal_x, normal_y, normal_z, curvature; };
struct PointNormal { float x, y, z, normal_x, normal_y, normal_z, curvature; };
struct PointXYZRGB { float x, y, z; unsigned char r, g, b; };
struct PointXYZRGBNormal { float x, y, z, normal_x, normal_y, normal_z, curvature; unsigned char r, g, b; };
}  // namespace pcl
