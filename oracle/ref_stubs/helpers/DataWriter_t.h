/* VTK-free stand-in for the reference's DataWriter_t, so the reference CPU
 * path compiles as a test checker (oracle/_ref) without VTK. Writing is a
 * no-op; the checker reads solution arrays straight from the mesh. */
#ifndef NDG_HELPERS_DATAWRITER_T_H
#define NDG_HELPERS_DATAWRITER_T_H

#include "helpers/float_types.h"
#include <filesystem>
#include <string>
#include <vector>

namespace SEM { namespace Helpers {
    class DataWriter_t {
        public:
            explicit DataWriter_t(std::filesystem::path) {}

            auto write_data(size_t, size_t, deviceFloat, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&) const -> void {}

            auto write_complete_data(size_t, size_t, deviceFloat, int, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<int>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<int>&, const std::vector<int>&, const std::vector<int>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<deviceFloat>&, const std::vector<int>&, const std::vector<int>&) const -> void {}
    };
}}

#endif
