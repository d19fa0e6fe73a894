// Solution output files: the role of the reference's DataWriter_t
// (src/helpers/DataWriter_t.cpp:18-546, include/helpers/DataWriter_t.h),
// written without VTK.
//
// Per output time, the reference's vtkXMLPUnstructuredGridWriter produces a
// parallel unstructured grid: a summary file named
// <stem>_t<time, 9 decimals, '.' -> '_'>s<ext> that lists one piece per
// rank, and the piece itself. Here the summary (PUnstructuredGrid) is
// written under that name and the single piece beside it as
// <same name without ext>_0.vtu, with the data arrays inline in base64
// (format="binary", UInt64 headers, no compression), which VTK and ParaView
// read. The grids and arrays follow the reference:
//   - the point grid: every element's n x n output points (x, y, 0), one
//     VTK_QUAD per grid cell with corners (i+1, j), (i+1, j+1), (i, j+1),
//     (i, j); point arrays Pressure, Velocity (2 components), and for the
//     complete output PressureDerivative, VelocityDerivative,
//     PressureAnalyticalError, VelocityAnalyticalError;
//   - the element grid (complete output only, <stem>_element...): one quad
//     per element through its output-grid corners (0, 0), (n-1, 0),
//     (n-1, n-1), (0, n-1); cell arrays N, Index, Status, Rotation, Rank,
//     PressureError, VelocityError (2), PressureSigma, VelocitySigma (2),
//     Refine, Coarsen, SplitLevel.
// The time series files <output>.series and <stem>_element<ext>.series are
// JSON {"file-series-version": "1.0", "files": [{"name", "time"}, ...]}
// printed with two-space indentation, created empty when the writer is
// made and extended at every output (DataWriter_t::create_time_series_file,
// add_time_series_to_file).
#include "../../include/ndg_b200.h"
#include "ndg_internal.hpp"

#include <array>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

namespace fs = std::filesystem;

struct ndg_writer {
    fs::path directory;
    std::string filename, extension;
    fs::path series, series_element;
    std::vector<std::pair<std::string, double>> files, files_element;
};

namespace ndg {
namespace {

template <typename F>
ndg_status writer_guarded(F&& f) {
    try {
        f();
        set_last_error("");
        return NDG_OK;
    } catch (const Error& e) {
        set_last_error(e.message);
        return e.status;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return NDG_ERR_INVALID_ARG;
    }
}

// A JSON number as a pretty-printing JSON library writes a double: the
// shortest digits that round-trip, in fixed notation when the decimal point
// falls within 15 digits of them (with ".0" after integral values) or up to
// 4 zeros after the point, otherwise d.ddde+XX with a two-digit exponent.
std::string json_number(double v) {
    if (!std::isfinite(v)) return "null";
    if (v == 0.0) return std::signbit(v) ? "-0.0" : "0.0";
    std::string out = v < 0 ? "-" : "";
    char buf[64];
    const auto res = std::to_chars(buf, buf + sizeof(buf), std::fabs(v), std::chars_format::scientific);
    const std::string sci(buf, res.ptr);
    const size_t epos = sci.find('e');
    std::string digits = sci.substr(0, 1) + (epos > 2 ? sci.substr(2, epos - 2) : "");
    const int exp10 = std::stoi(sci.substr(epos + 1));
    const int k = static_cast<int>(digits.size());
    const int n = exp10 + 1;  // position of the decimal point after the first n digits
    if (k <= n && n <= 15) {
        out += digits + std::string(static_cast<size_t>(n - k), '0') + ".0";
    } else if (0 < n && n <= 15) {
        out += digits.substr(0, static_cast<size_t>(n)) + "." + digits.substr(static_cast<size_t>(n));
    } else if (-4 < n && n <= 0) {
        out += "0." + std::string(static_cast<size_t>(-n), '0') + digits;
    } else {
        out += digits.substr(0, 1);
        if (k > 1) out += "." + digits.substr(1);
        const int e = n - 1;
        char eb[16];
        std::snprintf(eb, sizeof(eb), "e%c%02d", e < 0 ? '-' : '+', e < 0 ? -e : e);
        out += eb;
    }
    return out;
}

std::string json_string(const std::string& s) {
    std::string out = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') {
            out += '\\';
            out += c;
        } else if (static_cast<unsigned char>(c) < 0x20) {
            char b[8];
            std::snprintf(b, sizeof(b), "\\u%04x", static_cast<unsigned>(static_cast<unsigned char>(c)));
            out += b;
        } else {
            out += c;
        }
    }
    return out + "\"";
}

void write_series(const fs::path& path, const std::vector<std::pair<std::string, double>>& files) {
    std::ofstream o(path, std::ios::trunc);
    if (!o) fail(NDG_ERR_INVALID_ARG, "cannot write " + path.string());
    o << "{\n  \"file-series-version\": \"1.0\",\n  \"files\": ";
    if (files.empty()) {
        o << "[]\n}\n";
        return;
    }
    o << "[\n";
    for (size_t i = 0; i < files.size(); ++i) {
        o << "    {\n      \"name\": " << json_string(files[i].first) << ",\n      \"time\": " << json_number(files[i].second) << "\n    }"
          << (i + 1 < files.size() ? ",\n" : "\n");
    }
    o << "  ]\n}\n";
}

std::string base64(const uint8_t* data, size_t n) {
    static const char* tbl = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    std::string out;
    out.reserve((n + 2) / 3 * 4);
    size_t i = 0;
    for (; i + 2 < n; i += 3) {
        const uint32_t w = (uint32_t(data[i]) << 16) | (uint32_t(data[i + 1]) << 8) | data[i + 2];
        out += tbl[(w >> 18) & 63];
        out += tbl[(w >> 12) & 63];
        out += tbl[(w >> 6) & 63];
        out += tbl[w & 63];
    }
    if (i < n) {
        const uint32_t w = (uint32_t(data[i]) << 16) | (i + 1 < n ? uint32_t(data[i + 1]) << 8 : 0u);
        out += tbl[(w >> 18) & 63];
        out += tbl[(w >> 12) & 63];
        out += (i + 1 < n) ? tbl[(w >> 6) & 63] : '=';
        out += '=';
    }
    return out;
}

// One data array in VTK's inline binary form: base64 of a UInt64 byte count followed by the raw values.
template <typename T>
std::string data_array(const char* type, const char* name, int components, const std::vector<T>& values) {
    std::vector<uint8_t> raw(sizeof(uint64_t) + values.size() * sizeof(T));
    const uint64_t bytes = values.size() * sizeof(T);
    std::memcpy(raw.data(), &bytes, sizeof(bytes));
    if (!values.empty()) std::memcpy(raw.data() + sizeof(bytes), values.data(), bytes);
    std::ostringstream s;
    s << "        <DataArray type=\"" << type << "\"";
    if (name) s << " Name=\"" << name << "\"";
    if (components > 1) s << " NumberOfComponents=\"" << components << "\"";
    s << " format=\"binary\">\n          " << base64(raw.data(), raw.size()) << "\n        </DataArray>\n";
    return s.str();
}

struct Array {
    std::string text;       // the piece's DataArray element
    std::string summary;    // the PDataArray element of the summary file
};

template <typename T>
Array make_array(const char* type, const char* name, int components, const std::vector<T>& values) {
    std::ostringstream p;
    p << "      <PDataArray type=\"" << type << "\" Name=\"" << name << "\"";
    if (components > 1) p << " NumberOfComponents=\"" << components << "\"";
    p << "/>\n";
    return {data_array(type, name, components, values), p.str()};
}

// Writes summary file `path` and its piece for a grid of quads.
void write_grid(const fs::path& path, const std::vector<double>& points_xyz, const std::vector<int64_t>& connectivity,
                const std::vector<Array>& point_data, const std::vector<Array>& cell_data) {
    const int64_t n_points = static_cast<int64_t>(points_xyz.size() / 3);
    const int64_t n_cells = static_cast<int64_t>(connectivity.size() / 4);
    fs::path piece = path;
    piece.replace_extension("");
    const std::string piece_name = piece.filename().string() + "_0.vtu";
    const fs::path piece_path = path.parent_path() / piece_name;
    {
        std::vector<int64_t> offsets(static_cast<size_t>(n_cells));
        for (int64_t c = 0; c < n_cells; ++c) offsets[static_cast<size_t>(c)] = 4 * (c + 1);
        const std::vector<uint8_t> types(static_cast<size_t>(n_cells), 9);  // VTK_QUAD
        std::ofstream o(piece_path, std::ios::trunc);
        if (!o) fail(NDG_ERR_INVALID_ARG, "cannot write " + piece_path.string());
        o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
          << "  <UnstructuredGrid>\n    <Piece NumberOfPoints=\"" << n_points << "\" NumberOfCells=\"" << n_cells << "\">\n";
        o << "      <PointData>\n";
        for (const auto& a : point_data) o << a.text;
        o << "      </PointData>\n      <CellData>\n";
        for (const auto& a : cell_data) o << a.text;
        o << "      </CellData>\n      <Points>\n" << data_array("Float64", "Points", 3, points_xyz) << "      </Points>\n      <Cells>\n"
          << data_array("Int64", "connectivity", 1, connectivity) << data_array("Int64", "offsets", 1, offsets)
          << data_array("UInt8", "types", 1, types) << "      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n";
        if (!o) fail(NDG_ERR_INVALID_ARG, "write failed: " + piece_path.string());
    }
    std::ofstream o(path, std::ios::trunc);
    if (!o) fail(NDG_ERR_INVALID_ARG, "cannot write " + path.string());
    o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"PUnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
      << "  <PUnstructuredGrid GhostLevel=\"0\">\n    <PPointData>\n";
    for (const auto& a : point_data) o << a.summary;
    o << "    </PPointData>\n    <PCellData>\n";
    for (const auto& a : cell_data) o << a.summary;
    o << "    </PCellData>\n    <PPoints>\n      <PDataArray type=\"Float64\" Name=\"Points\" NumberOfComponents=\"3\"/>\n    </PPoints>\n"
      << "    <Piece Source=\"" << piece_name << "\"/>\n  </PUnstructuredGrid>\n</VTKFile>\n";
    if (!o) fail(NDG_ERR_INVALID_ARG, "write failed: " + path.string());
}

std::string time_string(double time) {
    char b[64];
    std::snprintf(b, sizeof(b), "_t%.9fs", time);
    std::string s(b);
    for (char& c : s)
        if (c == '.') c = '_';
    return s;
}

std::vector<double> interleave(const double* a, const double* b, int64_t n) {
    std::vector<double> out(static_cast<size_t>(2 * n), 0.0);
    for (int64_t i = 0; i < n; ++i) {
        out[static_cast<size_t>(2 * i)] = a ? a[i] : 0.0;
        out[static_cast<size_t>(2 * i + 1)] = b ? b[i] : 0.0;
    }
    return out;
}

template <typename T>
std::vector<T> copy_or_zero(const T* a, int64_t n) {
    return a ? std::vector<T>(a, a + n) : std::vector<T>(static_cast<size_t>(n), T{});
}

}  // namespace
}  // namespace ndg

using namespace ndg;

extern "C" {

ndg_status ndg_writer_create(const char* output_filename, ndg_writer** out) {
    return writer_guarded([&] {
        if (!output_filename || !out) fail(NDG_ERR_INVALID_ARG, "NULL argument");
        const fs::path p(output_filename);
        auto* w = new ndg_writer();
        w->directory = p.parent_path();
        w->filename = p.stem().string();
        w->extension = p.extension().string();
        w->series = p;
        w->series += ".series";
        w->series_element = w->directory / (w->filename + "_element" + w->extension + ".series");
        try {
            write_series(w->series, w->files);
            write_series(w->series_element, w->files_element);
        } catch (...) {
            delete w;
            throw;
        }
        *out = w;
    });
}

ndg_status ndg_writer_destroy(ndg_writer* writer) {
    delete writer;
    return NDG_OK;
}

ndg_status ndg_writer_write_arrays(ndg_writer* w, double time, int64_t n_elements, int64_t n_interp, const ndg_output_arrays* a) {
    return writer_guarded([&] {
        if (!w || !a) fail(NDG_ERR_INVALID_ARG, "NULL argument");
        if (n_elements < 0 || n_interp < 2) fail(NDG_ERR_INVALID_ARG, "need n_elements >= 0 and n_interp >= 2");
        if (!a->x || !a->y || !a->p || !a->u || !a->v) fail(NDG_ERR_INVALID_ARG, "x, y, p, u and v are required");
        const int64_t P = n_interp, PP = P * P, n_points = n_elements * PP;
        std::vector<double> xyz(static_cast<size_t>(3 * n_points));
        for (int64_t i = 0; i < n_points; ++i) {
            xyz[static_cast<size_t>(3 * i)] = a->x[i];
            xyz[static_cast<size_t>(3 * i + 1)] = a->y[i];
            xyz[static_cast<size_t>(3 * i + 2)] = 0.0;
        }
        std::vector<int64_t> conn;
        conn.reserve(static_cast<size_t>(4 * n_elements * (P - 1) * (P - 1)));
        for (int64_t e = 0; e < n_elements; ++e) {
            const int64_t o = e * PP;
            for (int64_t i = 0; i + 1 < P; ++i)
                for (int64_t j = 0; j + 1 < P; ++j) {
                    conn.push_back(o + (i + 1) * P + j);
                    conn.push_back(o + (i + 1) * P + j + 1);
                    conn.push_back(o + i * P + j + 1);
                    conn.push_back(o + i * P + j);
                }
        }
        std::vector<Array> pd;
        pd.push_back(make_array("Float64", "Pressure", 1, std::vector<double>(a->p, a->p + n_points)));
        pd.push_back(make_array("Float64", "Velocity", 2, interleave(a->u, a->v, n_points)));
        const std::string ts = time_string(time);
        const std::string name = w->filename + ts + w->extension;
        if (!a->complete) {
            write_grid(w->directory / name, xyz, conn, pd, {});
            w->files.emplace_back(name, time);
            write_series(w->series, w->files);
            return;
        }
        pd.push_back(make_array("Float64", "PressureDerivative", 1, copy_or_zero(a->dp_dt, n_points)));
        pd.push_back(make_array("Float64", "VelocityDerivative", 2, interleave(a->du_dt, a->dv_dt, n_points)));
        pd.push_back(make_array("Float64", "PressureAnalyticalError", 1, copy_or_zero(a->p_analytical_error, n_points)));
        pd.push_back(make_array("Float64", "VelocityAnalyticalError", 2, interleave(a->u_analytical_error, a->v_analytical_error, n_points)));

        std::vector<double> exyz(static_cast<size_t>(12 * n_elements));
        std::vector<int64_t> econn(static_cast<size_t>(4 * n_elements));
        const int64_t corner[4] = {0, (P - 1) * P, (P - 1) * P + (P - 1), P - 1};
        for (int64_t e = 0; e < n_elements; ++e)
            for (int c = 0; c < 4; ++c) {
                const int64_t src = e * PP + corner[c];
                exyz[static_cast<size_t>(12 * e + 3 * c)] = a->x[src];
                exyz[static_cast<size_t>(12 * e + 3 * c + 1)] = a->y[src];
                exyz[static_cast<size_t>(12 * e + 3 * c + 2)] = 0.0;
                econn[static_cast<size_t>(4 * e + c)] = 4 * e + c;
            }
        std::vector<uint64_t> index(static_cast<size_t>(n_elements));
        for (int64_t e = 0; e < n_elements; ++e) index[static_cast<size_t>(e)] = static_cast<uint64_t>(e);
        std::vector<Array> cd;
        cd.push_back(make_array("Int32", "N", 1, copy_or_zero(a->N, n_elements)));
        cd.push_back(make_array("UInt64", "Index", 1, index));
        cd.push_back(make_array("Int32", "Status", 1, copy_or_zero(a->status, n_elements)));
        cd.push_back(make_array("Int32", "Rotation", 1, copy_or_zero(a->rotation, n_elements)));
        cd.push_back(make_array("Int32", "Rank", 1, std::vector<int32_t>(static_cast<size_t>(n_elements), a->rank)));
        cd.push_back(make_array("Float64", "PressureError", 1, copy_or_zero(a->p_error, n_elements)));
        cd.push_back(make_array("Float64", "VelocityError", 2, interleave(a->u_error, a->v_error, n_elements)));
        cd.push_back(make_array("Float64", "PressureSigma", 1, copy_or_zero(a->p_sigma, n_elements)));
        cd.push_back(make_array("Float64", "VelocitySigma", 2, interleave(a->u_sigma, a->v_sigma, n_elements)));
        cd.push_back(make_array("Int32", "Refine", 1, copy_or_zero(a->refine, n_elements)));
        cd.push_back(make_array("Int32", "Coarsen", 1, copy_or_zero(a->coarsen, n_elements)));
        cd.push_back(make_array("Int32", "SplitLevel", 1, copy_or_zero(a->split_level, n_elements)));

        const std::string ename = w->filename + "_element" + ts + w->extension;
        write_grid(w->directory / name, xyz, conn, pd, {});
        write_grid(w->directory / ename, exyz, econn, {}, cd);
        w->files.emplace_back(name, time);
        w->files_element.emplace_back(ename, time);
        write_series(w->series, w->files);
        write_series(w->series_element, w->files_element);
    });
}

}  // extern "C"
