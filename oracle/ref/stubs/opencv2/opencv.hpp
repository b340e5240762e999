// Stand-in for opencv2/opencv.hpp, written for compiling the reference's index kernels in place
// (oracle/ref/Makefile): the reference's visualisation headers declare functions over cv::Mat,
// which the checked kernels never call.
#pragma once
// the standard headers the real one brings in and the reference relies on
#include <map>
#include <string>
#include <vector>

namespace cv {
class Mat {};
constexpr int IMREAD_ANYCOLOR = 4;
constexpr int IMREAD_ANYDEPTH = 2;
}  // namespace cv
