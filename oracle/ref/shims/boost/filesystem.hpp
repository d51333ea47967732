// Stand-in for the few boost::filesystem calls made by the reference's
// src/core/filesystem.cpp (exists, path queries, create/rename/remove).
// std::filesystem provides the same operations with the same meaning.
#pragma once
#include <filesystem>
#include <cassert>   // boost/filesystem.hpp brings this in transitively
namespace boost { namespace filesystem { using namespace std::filesystem; } }
