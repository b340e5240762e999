// Stand-in for boost/filesystem.hpp, written for compiling the reference's index kernels in
// place (oracle/ref/Makefile): the reference names boost::filesystem::path only.
#pragma once
#include <filesystem>

namespace boost {
namespace filesystem {
using path = std::filesystem::path;
}
}  // namespace boost
