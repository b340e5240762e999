// Stand-in for pcl/io/pcd_io.h, written for compiling the reference's index kernels in place
// (oracle/ref/Makefile): a visualisation helper the checked kernels never call saves a cloud.
#pragma once
#include <string>

#include "../point_cloud.h"

namespace pcl {
namespace io {
template <typename PointT>
int savePCDFileBinary(const std::string &, const PointCloud<PointT> &) {
    return -1;
}
}  // namespace io
}  // namespace pcl
