// Stand-in for nlohmann/json.hpp, written for compiling the reference's index kernels in place
// (oracle/ref/Makefile): the reference's graph visualiser, an inline header function the checked
// kernels never call, assigns values to keys and streams the object.  Nothing is stored.
#pragma once
#include <iomanip>
#include <ostream>
#include <string>

namespace nlohmann {
class json {
public:
    json() = default;
    template <typename T>
    json(const T &) {}
    json &operator[](const char *) { return *this; }
    json &operator[](const std::string &) { return *this; }
    template <typename T>
    json &operator=(const T &) { return *this; }
    friend std::ostream &operator<<(std::ostream &o, const json &) { return o; }
};
}  // namespace nlohmann
