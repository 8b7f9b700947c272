// ot_fs_shim.hpp -- force-included (-include) when the reference sources are
// compiled into oracle/_ref/.  The reference declares
//   namespace std { namespace filesystem = experimental::filesystem; }
// which collides with the std::filesystem namespace that libstdc++ 13
// forward-declares in C++17 mode.  Every standard header is pulled in first,
// std::filesystem is given a second name, and the token `filesystem` is then
// renamed to that name, so the reference's alias line becomes a harmless
// re-declaration.  The reference's own files are compiled unmodified.
#pragma once
#include <bits/stdc++.h>
#include <filesystem>
namespace std {
namespace experimental { namespace otg_fs_ = ::std::filesystem; }
namespace otg_fs_ = ::std::filesystem;
}
#define filesystem otg_fs_
