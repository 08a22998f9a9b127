// Array files on the host: MetaImage (.mha with the data after the header, .mhd with a separate
// raw file), Dennerlein (.den) and headerless raw binaries, read into and written from plain
// numeric arrays. Replaces GCT::IO's readers (src/cpp/io/file_reader/array_file_reader.cpp,
// meta_img_reader.cpp:10-165, den_file_reader.cpp, raw_data_file_reader.cpp; series of files by
// src/cpp/io/file_utils.cpp:7-27) and writers (src/cpp/io/file_writer/meta_img_file_writer.{h,cpp},
// den_file_writer.h, raw_data_file_writer.h). The header grammar and the checks follow those
// files; where the reference reads out of bounds or accepts a short file, this code reports an
// error instead (noted at each place).
#include "../../include/gct_fdk.h"
#include "plan.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace fs = std::filesystem;

namespace gct {
namespace {

size_t elem_bytes(int type)
{
    switch (type) {
        case GCT_T_UINT8:
        case GCT_T_INT8: return 1;
        case GCT_T_UINT16:
        case GCT_T_INT16: return 2;
        case GCT_T_UINT32:
        case GCT_T_INT32:
        case GCT_T_FLOAT: return 4;
        case GCT_T_UINT64:
        case GCT_T_INT64:
        case GCT_T_DOUBLE: return 8;
        default: fail(GCT_ERR_INVALID_ARG, "unknown element type " + std::to_string(type));
    }
    return 0;
}

// MetaImage ElementType names (meta_img_reader.cpp setTypeMap; meta_img_file_writer.cpp typeStr).
const char *meta_type_name(int type)
{
    static const char *names[] = {"MET_UCHAR", "MET_CHAR",  "MET_USHORT",     "MET_SHORT",     "MET_UINT",
                                  "MET_INT",   "MET_ULONG_LONG", "MET_LONG_LONG", "MET_FLOAT", "MET_DOUBLE"};
    elem_bytes(type);  // validates
    return names[type];
}
int meta_type_of(const std::string &name)
{
    for (int t = GCT_T_UINT8; t <= GCT_T_DOUBLE; ++t)
        if (name == meta_type_name(t)) return t;
    return -1;
}

std::string trim(const std::string &s)
{
    const char *ws = " \t\r\n";
    const size_t b = s.find_first_not_of(ws);
    if (b == std::string::npos) return "";
    return s.substr(b, s.find_last_not_of(ws) - b + 1);
}

uint64_t num_elems(const gct_array_metadata &md)
{
    return static_cast<uint64_t>(md.num_rows) * md.num_cols * md.num_slices;
}

// getAllFiles (file_utils.cpp:7-27): every file under the directory of `filename` (recursively)
// with its extension and its size, in sorted order.
std::vector<std::string> series_files(const std::string &filename)
{
    const fs::path p{filename};
    if (!fs::exists(p)) fail(GCT_ERR_INVALID_ARG, "File " + filename + " is not found.");
    const fs::path dir = p.parent_path().empty() ? fs::path{"."} : p.parent_path();
    const auto ext = p.extension();
    const auto size = fs::file_size(p);
    std::vector<std::string> files;
    for (const auto &e : fs::recursive_directory_iterator(dir))
        if (e.is_regular_file() && e.path().extension() == ext && fs::file_size(e.path()) == size)
            files.push_back(e.path().string());
    std::sort(files.begin(), files.end());
    return files;
}

// readDataFromBinFile (array_file_reader.cpp): the file, less `skip` leading bytes, must hold
// exactly the bytes of the metadata.
void read_bin(const std::string &filename, size_t skip, size_t bytes, unsigned char *dst)
{
    std::ifstream f(filename, std::ios::binary);
    if (!f) fail(GCT_ERR_INVALID_ARG, "File " + filename + " cannot be opened for reading data.");
    f.seekg(0, std::ios::end);
    const size_t size = static_cast<size_t>(f.tellg());
    if (skip > size)
        fail(GCT_ERR_INVALID_ARG, "Error during the reading of file " + filename + ": the file holds " +
                                      std::to_string(size) + " bytes, " + std::to_string(skip) + " are to be skipped.");
    if (bytes != size - skip)
        fail(GCT_ERR_INVALID_ARG, "Error during the reading of file " + filename + ": the file holds " +
                                      std::to_string(size - skip) + " data bytes, the metadata needs " +
                                      std::to_string(bytes) + ".");
    f.seekg(static_cast<std::streamoff>(skip), std::ios::beg);
    f.read(reinterpret_cast<char *>(dst), static_cast<std::streamsize>(bytes));
    if (!f) fail(GCT_ERR_INVALID_ARG, "Error during the reading of file " + filename + ".");
}

// ---- MetaImage --------------------------------------------------------------------------------

// readElementDataFile: the value of the first line holding "ElementDataFile".
std::string meta_data_file(const std::string &header)
{
    std::ifstream f(header);
    std::string line;
    while (std::getline(f, line))
        if (line.find("ElementDataFile") != std::string::npos) return trim(line.substr(line.find('=') + 1));
    return "";
}

// readMetadata: DimSize (columns, rows[, slices]) and ElementType, up to the LOCAL data line.
// A DimSize with fewer than two entries is an error here (the reference indexes past it).
gct_array_metadata meta_metadata(const std::string &header)
{
    std::ifstream f(header);
    if (!f) fail(GCT_ERR_INVALID_ARG, "File " + header + " cannot be opened.");
    gct_array_metadata md{1u, 1u, 1u, GCT_T_UINT8};
    bool have_type = false;
    std::string line;
    while (std::getline(f, line)) {
        if (line.find("ElementDataFile = LOCAL") != std::string::npos) break;
        if (line.find("DimSize ") != std::string::npos) {
            std::stringstream ss{line.substr(line.find('=') + 1)};
            std::vector<long long> dims;
            std::string w;
            while (ss >> w) dims.push_back(std::stoll(w));
            if (dims.size() < 2 || dims.size() > 3)
                fail(GCT_ERR_INVALID_ARG, "Error during reading meta image file " + header + ": DimSize needs 2 or 3 values");
            for (long long d : dims)
                if (d <= 0 || d > 0xffffffffll)
                    fail(GCT_ERR_INVALID_ARG, "Error during reading meta image file " + header + ": bad DimSize");
            md.num_cols = static_cast<uint32_t>(dims[0]);
            md.num_rows = static_cast<uint32_t>(dims[1]);
            if (dims.size() == 3) md.num_slices = static_cast<uint32_t>(dims[2]);
        }
        if (line.find("ElementType ") != std::string::npos) {
            const std::string v = trim(line.substr(line.find('=') + 1));
            const int t = meta_type_of(v);
            if (t < 0)
                fail(GCT_ERR_INVALID_ARG,
                     "Error during reading meta image file " + header + "\n" + v + " is not a valid ElementType");
            md.type = t;
            have_type = true;
        }
    }
    if (!have_type) fail(GCT_ERR_INVALID_ARG, "Error during reading meta image file " + header + ": no ElementType");
    return md;
}

// Data of a file with its header (readDataBytesMHAFile): the bytes after the line
// "ElementDataFile = LOCAL". A short file is an error here (the reference leaves zeros).
void read_mha_data(const std::string &filename, size_t bytes, unsigned char *dst)
{
    std::ifstream f(filename, std::ios::binary);
    if (!f) fail(GCT_ERR_INVALID_ARG, "File " + filename + " cannot be opened for reading data.");
    std::string line;
    bool found = false;
    while (std::getline(f, line))
        if (line == "ElementDataFile = LOCAL") {
            found = true;
            break;
        }
    if (!found) fail(GCT_ERR_INVALID_ARG, "File " + filename + " has no \"ElementDataFile = LOCAL\" line.");
    f.read(reinterpret_cast<char *>(dst), static_cast<std::streamsize>(bytes));
    if (static_cast<size_t>(f.gcount()) != bytes)
        fail(GCT_ERR_INVALID_ARG, "File " + filename + " holds fewer data bytes than its header needs.");
}

// ---- Dennerlein -------------------------------------------------------------------------------

// Header of three uint16 (rows, columns, slices); the element type follows from the file size
// (den_file_reader.cpp dataType: 1 byte uint8, 2 uint16, 4 float, 8 double, otherwise uint8).
gct_array_metadata den_metadata(const std::string &filename)
{
    std::ifstream f(filename, std::ios::binary);
    if (!f) fail(GCT_ERR_INVALID_ARG, "File " + filename + " cannot be opened.");
    uint16_t h[3] = {0, 0, 0};
    f.read(reinterpret_cast<char *>(h), sizeof(h));
    if (!f) fail(GCT_ERR_INVALID_ARG, "File " + filename + " is shorter than a Dennerlein header.");
    gct_array_metadata md{h[0], h[1], h[2], GCT_T_UINT8};
    const uint64_t n = num_elems(md);
    const uint64_t data = fs::file_size(filename) - sizeof(h);
    const uint64_t es = n ? data / n : 0;
    md.type = es == 2 ? GCT_T_UINT16 : es == 4 ? GCT_T_FLOAT : es == 8 ? GCT_T_DOUBLE : GCT_T_UINT8;
    return md;
}

// ---- reading ----------------------------------------------------------------------------------

struct Source {
    gct_array_metadata md{};
    std::vector<std::string> files;  // data files, one per series member
    int kind = 0;                    // 0 raw bytes at `skip`, 1 MetaImage with its header
    size_t skip = 0;
};

Source open_source(const std::string &filename, int format, bool series, const gct_array_metadata *raw_md)
{
    if (!fs::exists(fs::path{filename})) fail(GCT_ERR_INVALID_ARG, "File " + filename + " is not found.");
    Source s;
    std::string data_file = filename;
    switch (format) {
        case GCT_FILE_META_IMAGE: {
            s.md = meta_metadata(filename);
            const std::string df = meta_data_file(filename);
            if (df == "LOCAL") {
                s.kind = 1;
            } else {
                const fs::path raw = fs::path{filename}.parent_path() / df;
                if (df.empty() || !fs::exists(raw))
                    fail(GCT_ERR_INVALID_ARG, "Data filename " + raw.string() +
                                                  " is not found.\nHeader and data files should be in the same directory.");
                data_file = raw.string();
            }
            break;
        }
        case GCT_FILE_DEN:
            s.md = den_metadata(filename);
            s.skip = 3 * sizeof(uint16_t);
            break;
        case GCT_FILE_RAW:
            if (!raw_md) fail(GCT_ERR_INVALID_ARG, "raw files need their metadata");
            s.md = *raw_md;
            elem_bytes(s.md.type);
            break;
        default: fail(GCT_ERR_INVALID_ARG, "unknown file format " + std::to_string(format));
    }
    s.files = series ? series_files(data_file) : std::vector<std::string>{data_file};
    return s;
}

template <class In, class Out>
void convert_n(const unsigned char *src, Out *dst, uint64_t n)
{
    In v;
    for (uint64_t i = 0; i < n; ++i) {
        std::memcpy(&v, src + i * sizeof(In), sizeof(In));
        dst[i] = static_cast<Out>(v);
    }
}

template <class Out>
void convert_from(int in_type, const unsigned char *src, Out *dst, uint64_t n)
{
    switch (in_type) {
        case GCT_T_UINT8: convert_n<uint8_t>(src, dst, n); break;
        case GCT_T_INT8: convert_n<int8_t>(src, dst, n); break;
        case GCT_T_UINT16: convert_n<uint16_t>(src, dst, n); break;
        case GCT_T_INT16: convert_n<int16_t>(src, dst, n); break;
        case GCT_T_UINT32: convert_n<uint32_t>(src, dst, n); break;
        case GCT_T_INT32: convert_n<int32_t>(src, dst, n); break;
        case GCT_T_UINT64: convert_n<uint64_t>(src, dst, n); break;
        case GCT_T_INT64: convert_n<int64_t>(src, dst, n); break;
        case GCT_T_FLOAT: convert_n<float>(src, dst, n); break;
        default: convert_n<double>(src, dst, n); break;
    }
}

// convertData (array_file_reader.h): every element static_cast to the output type.
void convert(int in_type, const unsigned char *src, int out_type, void *dst, uint64_t n)
{
    switch (out_type) {
        case GCT_T_UINT8: convert_from(in_type, src, static_cast<uint8_t *>(dst), n); break;
        case GCT_T_INT8: convert_from(in_type, src, static_cast<int8_t *>(dst), n); break;
        case GCT_T_UINT16: convert_from(in_type, src, static_cast<uint16_t *>(dst), n); break;
        case GCT_T_INT16: convert_from(in_type, src, static_cast<int16_t *>(dst), n); break;
        case GCT_T_UINT32: convert_from(in_type, src, static_cast<uint32_t *>(dst), n); break;
        case GCT_T_INT32: convert_from(in_type, src, static_cast<int32_t *>(dst), n); break;
        case GCT_T_UINT64: convert_from(in_type, src, static_cast<uint64_t *>(dst), n); break;
        case GCT_T_INT64: convert_from(in_type, src, static_cast<int64_t *>(dst), n); break;
        case GCT_T_FLOAT: convert_from(in_type, src, static_cast<float *>(dst), n); break;
        case GCT_T_DOUBLE: convert_from(in_type, src, static_cast<double *>(dst), n); break;
        default: fail(GCT_ERR_INVALID_ARG, "unknown element type " + std::to_string(out_type));
    }
}

// ---- writing ----------------------------------------------------------------------------------

// isWritable (file_utils.h) of the parent directory; a bare file name means the working
// directory here (the reference rejects it: its parent path is empty).
std::ofstream open_for_write(const std::string &filename, const char *what)
{
    const fs::path p{filename};
    const fs::path dir = p.parent_path().empty() ? fs::path{"."} : p.parent_path();
    std::error_code ec;
    const auto st = fs::status(dir, ec);
    if (ec || !fs::is_directory(st) || (st.permissions() & fs::perms::owner_write) == fs::perms::none)
        fail(GCT_ERR_INVALID_ARG, std::string("Error during the writing of ") + what + " " + filename +
                                      "\nParent directory is not writable.");
    std::ofstream f(filename, std::ios::binary);
    if (!f) fail(GCT_ERR_INVALID_ARG, std::string("Error during the writing of ") + what + " " + filename +
                                          "\nFile cannot be opened.");
    return f;
}

void write_bytes(std::ofstream &f, const void *data, size_t bytes, const std::string &filename)
{
    f.write(static_cast<const char *>(data), static_cast<std::streamsize>(bytes));
    if (!f) fail(GCT_ERR_INVALID_ARG, "Error during the writing of " + filename);
}

std::string lower(std::string s)
{
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
    return s;
}

// std::to_string of a float (the reference's header arrays): "%f" of the value.
std::string float_str(float v)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%f", static_cast<double>(v));
    return buf;
}

}  // namespace
}  // namespace gct

using gct::fail;

extern "C" {

gct_status gct_array_read_metadata(const char *filename, int32_t format, gct_array_metadata *md)
{
    return guarded([&] {
        if (!filename || !md) fail(GCT_ERR_INVALID_ARG, "NULL argument");
        const gct::Source s = gct::open_source(filename, format, false, format == GCT_FILE_RAW ? md : nullptr);
        *md = s.md;
    });
}

gct_status gct_array_read(const char *filename, int32_t format, int32_t series, const gct_array_metadata *raw_md,
                          int32_t out_type, void *out, uint64_t out_count, uint64_t *count)
{
    return guarded([&] {
        if (!filename) fail(GCT_ERR_INVALID_ARG, "NULL file name");
        const gct::Source s = gct::open_source(filename, format, series != 0, raw_md);
        const uint64_t per_file = gct::num_elems(s.md);
        const uint64_t total = per_file * s.files.size();
        if (count) *count = total;
        if (!out) return;  // size query
        gct::elem_bytes(out_type);
        if (out_count != total)
            fail(GCT_ERR_INVALID_ARG, "output holds " + std::to_string(out_count) + " elements, the file(s) " +
                                          std::to_string(total));
        const size_t in_es = gct::elem_bytes(s.md.type), out_es = gct::elem_bytes(out_type);
        std::vector<unsigned char> buf(static_cast<size_t>(per_file * in_es));
        for (size_t k = 0; k < s.files.size(); ++k) {
            if (s.kind == 1) gct::read_mha_data(s.files[k], buf.size(), buf.data());
            else gct::read_bin(s.files[k], s.skip, buf.size(), buf.data());
            gct::convert(s.md.type, buf.data(), out_type, static_cast<unsigned char *>(out) + k * per_file * out_es,
                         per_file);
        }
    });
}

gct_status gct_meta_image_write(const char *filename, uint32_t ndims, const uint32_t *dim_size, const float *spacing,
                                const float *offset, int32_t type, const void *data, uint64_t count)
{
    return guarded([&] {
        if (!filename || !dim_size || !spacing || !offset || (!data && count))
            fail(GCT_ERR_INVALID_ARG, "NULL argument");
        if (ndims < 1 || ndims > 3) fail(GCT_ERR_INVALID_ARG, "MetaImage files of 1 to 3 dimensions");
        uint64_t n = 1;
        for (uint32_t d = 0; d < ndims; ++d) n *= dim_size[d];
        if (n != count)
            fail(GCT_ERR_INVALID_ARG, std::string("Error during the writing of Meta image file ") + filename +
                                          "\nMismatch in the number of elements between data and metadata.");
        const char *tname = gct::meta_type_name(type);
        const size_t bytes = static_cast<size_t>(count) * gct::elem_bytes(type);
        std::ofstream f = gct::open_for_write(filename, "Meta image file");
        auto entry = [&](const std::string &tag, const std::string &val) { f << tag << " = " << val << "\n"; };
        auto arr = [&](auto get) {
            std::string s;
            for (uint32_t d = 0; d < ndims; ++d) s += (d ? " " : "") + get(d);
            return s;
        };
        entry("ObjectType", "Image");
        entry("NDims", std::to_string(ndims));
        entry("BinaryData", "True");
        entry("DimSize", arr([&](uint32_t d) { return std::to_string(dim_size[d]); }));
        entry("ElementSpacing", arr([&](uint32_t d) { return gct::float_str(spacing[d]); }));
        entry("Offset", arr([&](uint32_t d) { return gct::float_str(offset[d]); }));
        entry("ElementType", tname);
        entry("BinaryDataByteOrderMSB", "False");
        const fs::path p{filename};
        if (gct::lower(p.extension().string()) == ".mha") {
            entry("ElementDataFile", "LOCAL");
            gct::write_bytes(f, data, bytes, filename);
        } else {
            const std::string raw_name = p.stem().string() + ".raw";
            entry("ElementDataFile", raw_name);
            const std::string raw = (p.parent_path() / raw_name).string();
            std::ofstream r = gct::open_for_write(raw, "binary file");
            gct::write_bytes(r, data, bytes, raw);
        }
        if (!f) fail(GCT_ERR_INVALID_ARG, std::string("Error during the writing of ") + filename);
    });
}

gct_status gct_den_write(const char *filename, uint32_t num_rows, uint32_t num_cols, uint32_t num_slices,
                         int32_t type, const void *data, uint64_t count)
{
    return guarded([&] {
        if (!filename || (!data && count)) fail(GCT_ERR_INVALID_ARG, "NULL argument");
        if (num_rows > 0xffff || num_cols > 0xffff || num_slices > 0xffff)
            fail(GCT_ERR_INVALID_ARG, "Dennerlein dimensions are 16-bit");
        if (static_cast<uint64_t>(num_rows) * num_cols * num_slices != count)
            fail(GCT_ERR_INVALID_ARG, std::string("Error during the writing of Dennerlein file ") + filename +
                                          "\nMismatch in the number of elements between data and metadata.");
        const size_t bytes = static_cast<size_t>(count) * gct::elem_bytes(type);
        std::ofstream f = gct::open_for_write(filename, "Dennerlein file");
        const uint16_t h[3] = {static_cast<uint16_t>(num_rows), static_cast<uint16_t>(num_cols),
                               static_cast<uint16_t>(num_slices)};
        gct::write_bytes(f, h, sizeof(h), filename);
        gct::write_bytes(f, data, bytes, filename);
    });
}

gct_status gct_raw_write(const char *filename, int32_t type, const void *data, uint64_t count)
{
    return guarded([&] {
        if (!filename || (!data && count)) fail(GCT_ERR_INVALID_ARG, "NULL argument");
        const size_t bytes = static_cast<size_t>(count) * gct::elem_bytes(type);
        std::ofstream f = gct::open_for_write(filename, "binary file");
        gct::write_bytes(f, data, bytes, filename);
    });
}

}  // extern "C"
