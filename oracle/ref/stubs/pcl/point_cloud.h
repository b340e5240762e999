// Stand-in for pcl/point_cloud.h, written for compiling the reference's index kernels in place
// (oracle/ref/Makefile): the reference's headers name pcl::PointCloud<T> and its Ptr only.
#pragma once
#include <cstddef>
#include <memory>
#include <vector>

namespace pcl {
template <typename PointT>
class PointCloud {
public:
    using Ptr = std::shared_ptr<PointCloud<PointT>>;
    using ConstPtr = std::shared_ptr<const PointCloud<PointT>>;
    std::vector<PointT> points;
    void resize(std::size_t n) { points.resize(n); }
    std::size_t size() const { return points.size(); }
};
}  // namespace pcl
