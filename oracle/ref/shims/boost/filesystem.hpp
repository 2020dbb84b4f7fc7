// Boost.Filesystem is absent from this image. The reference uses it only to
// create and list output directories; std::filesystem does the same job.
#pragma once
#include <filesystem>
namespace boost {
namespace filesystem = std::filesystem;
namespace system { using error_code = std::error_code; }
}
