// C entry points over satidev/gct's own array-file readers and writers (src/cpp/io), compiled
// from the reference tree by oracle/build_ref.sh into oracle/_ref/libgct_ref_io.so.
// TEST INFRASTRUCTURE ONLY: tests/golden/make_io_golden.py uses it to write fixture files with
// the reference's writers and to record what the reference's readers return for them; nothing in
// the engine links or calls it.
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "cpp/io/file_reader/den_file_reader.h"
#include "cpp/io/file_reader/meta_img_reader.h"
#include "cpp/io/file_reader/raw_data_file_reader.h"
#include "cpp/io/file_writer/den_file_writer.h"
#include "cpp/io/file_writer/meta_img_file_writer.h"

namespace {
thread_local std::string g_err;

template <class F>
int guard(F &&f)
{
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}

template <class T>
int write_mi(const char *filename, int ndims, const unsigned *dims, const float *sp, const float *of, const T *data,
             size_t n)
{
    return guard([&] {
        std::vector<T> v(data, data + n);
        if (ndims == 2) {
            GCT::IO::ArrayFileWriter::MetaImgMetaData<2> md{{dims[0], dims[1]}, {sp[0], sp[1]}, {of[0], of[1]}};
            GCT::IO::ArrayFileWriter::write(md, v, filename);
        } else {
            GCT::IO::ArrayFileWriter::MetaImgMetaData<3> md{
                {dims[0], dims[1], dims[2]}, {sp[0], sp[1], sp[2]}, {of[0], of[1], of[2]}};
            GCT::IO::ArrayFileWriter::write(md, v, filename);
        }
    });
}

template <class T>
int write_den(const char *filename, unsigned rows, unsigned cols, unsigned slices, const T *data, size_t n)
{
    return guard([&] {
        std::vector<T> v(data, data + n);
        GCT::IO::ArrayFileWriter::DenMetaData md{static_cast<unsigned short>(rows), static_cast<unsigned short>(cols),
                                                 static_cast<unsigned short>(slices)};
        GCT::IO::ArrayFileWriter::write(md, v, filename);
    });
}
}  // namespace

extern "C" {

const char *ref_io_error() { return g_err.c_str(); }

// element kind: 0 float, 1 uint16, 2 int16, 3 double, 4 uint8
int ref_io_write_meta_image(const char *filename, int ndims, const unsigned *dims, const float *spacing,
                            const float *offset, int kind, const void *data, size_t n)
{
    switch (kind) {
        case 0: return write_mi(filename, ndims, dims, spacing, offset, static_cast<const float *>(data), n);
        case 1: return write_mi(filename, ndims, dims, spacing, offset, static_cast<const uint16_t *>(data), n);
        case 2: return write_mi(filename, ndims, dims, spacing, offset, static_cast<const int16_t *>(data), n);
        case 3: return write_mi(filename, ndims, dims, spacing, offset, static_cast<const double *>(data), n);
        default: return write_mi(filename, ndims, dims, spacing, offset, static_cast<const uint8_t *>(data), n);
    }
}

int ref_io_write_den(const char *filename, unsigned rows, unsigned cols, unsigned slices, int kind, const void *data,
                     size_t n)
{
    switch (kind) {
        case 0: return write_den(filename, rows, cols, slices, static_cast<const float *>(data), n);
        case 1: return write_den(filename, rows, cols, slices, static_cast<const uint16_t *>(data), n);
        case 3: return write_den(filename, rows, cols, slices, static_cast<const double *>(data), n);
        default: return write_den(filename, rows, cols, slices, static_cast<const uint8_t *>(data), n);
    }
}

// format: 0 MetaImage, 1 Dennerlein. Metadata as (rows, cols, slices, ArrayElemType).
int ref_io_read_metadata(const char *filename, int format, unsigned *md4)
{
    return guard([&] {
        GCT::IO::ArrayMetadata md{};
        if (format == 0) md = GCT::IO::MetaImgFileReader{filename}.readMetadata();
        else md = GCT::IO::DenFileReader{filename}.readMetadata();
        md4[0] = md.num_rows;
        md4[1] = md.num_cols;
        md4[2] = md.num_slices;
        md4[3] = static_cast<unsigned>(md.type);
    });
}

// readData<double> of the file (or its series); *count receives the element count, and up to
// `cap` elements are copied to out.
int ref_io_read_f64(const char *filename, int format, int series, double *out, size_t cap, size_t *count)
{
    return guard([&] {
        std::vector<double> v;
        if (format == 0) v = GCT::IO::MetaImgFileReader{filename, series != 0}.readData<double>();
        else v = GCT::IO::DenFileReader{filename, series != 0}.readData<double>();
        *count = v.size();
        std::memcpy(out, v.data(), sizeof(double) * std::min(cap, v.size()));
    });
}
}
