// Test-only stand-in for <boost/filesystem.hpp>: the one call the reference's
// command-line drivers make (cppcode/piece2aspl.cpp:51, box2aspl.cpp:51,
// main.cpp:53), boost::filesystem::file_size(path), following its documented
// behaviour (the size in bytes; an exception when the file cannot be read),
// implemented on std::filesystem.
#pragma once

#include <cstdint>
#include <filesystem>
#include <string>

namespace boost {
namespace filesystem {

using filesystem_error = std::filesystem::filesystem_error;

inline std::uintmax_t file_size(const std::string &path) { return std::filesystem::file_size(path); }

}  // namespace filesystem
}  // namespace boost
