// Parcel and field files in the reference's netCDF layout, written and read
// in the netCDF classic format (CDF-2, or CDF-5 when a variable exceeds the
// 4 GiB that CDF-2 allows).  The netCDF library reads both, so the reference
// can restart from these files (nf90_open, netcdf_utils.f90); the reference's
// own files are netCDF-4 (HDF5), which this reader does not parse.
//
// Layout (parcel_netcdf.f90:100-200, field_netcdf.f90:100-250,
// netcdf_writer.f90:374-600): global attributes file_type, ncells, extent,
// origin; an unlimited dimension t with a variable t (the time of each
// record); parcel files: dimensions n_parcels and world%size, record
// variables (t, n_parcels) x_position .. B23, and start_index, xlo, xhi, ylo,
// yhi over world%size; field files: dimensions x, y, z (nz+1 points), axis
// variables x, y, z and record variables (t, z, y, x) without halo rows.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace ncio {

// Thrown for unreadable files, missing variables and layout mismatches.
struct Error : std::runtime_error {
    explicit Error(const std::string& m) : std::runtime_error(m) {}
};

struct Box {
    int32_t ncells[3];
    double origin[3], extent[3];
};

struct Info {
    std::string file_type;
    Box box;
    int64_t n_parcels = 0;     // length of n_parcels (parcel files)
    int64_t n_steps = 0;       // records along t
    double t = 0.0;            // time of the last record
    int32_t zeta[2] = {0, 0};  // l_lower/upper_boundry_zeta_zero
    bool has_zeta = false;
    int version = 0;           // 1, 2 or 5
};

Info info(const std::string& path);

// Throws unless got and want have the same cells and (to 1e-12) extent and origin.
void check_box(const Box& got, const Box& want, const std::string& path);

// pos, vor: (3, n) interleaved per parcel; B: (5, n); vol, buoy, hum: (n).
// label, dil (may be null): the ENABLE_LABELS attributes, written as NC_INT64
// (which makes the file CDF-5) and NC_DOUBLE; labels below 2^53.
void write_parcels(const std::string& path, const Box& box, const int32_t zeta[2], double t, int64_t n,
                   const double* pos, const double* vor, const double* B, const double* vol,
                   const double* buoy, const double* hum, int force_version = 0,
                   const int64_t* label = nullptr, const double* dil = nullptr);

// Reads the first record (the reference writes one record per parcel file,
// read_chunk in parcel_netcdf.f90 reads record 1).  vor, buoy, hum that the
// file lacks are zero; at least one of them must be present and B11..B23,
// the positions and the volume always (parcel_netcdf.f90:600-700).
void read_parcels(const std::string& path, int64_t cap, int64_t* n, double* pos, double* vor, double* B,
                  double* vol, double* buoy, double* hum);

// One field of a field file: data in the library's field layout
// (nx, ny, nz+3), z fastest, rows z = -1 .. nz+1; rows 0 .. nz are written.
struct FieldOut {
    std::string name, long_name, unit;
    const double* data;
    bool integer;   // written as NC_INT (nparg, nsparg)
};
void write_fields(const std::string& path, const Box& box, const int32_t zeta[2], double t,
                  const std::vector<FieldOut>& fields, int force_version = 0);

// Reads record `step` (0-based; -1: the last) of a field variable into the
// field layout, rows 0 .. nz; other rows are left as they are.  Returns false
// if the file has no such variable.
bool read_field(const std::string& path, const std::string& name, int64_t step, const Box& expect, double* out);

// Record `record` (ignored for a fixed-size variable) of any numeric
// variable, converted to double, in C order; returns its element count and
// writes it to out when it fits cap.
int64_t read_variable(const std::string& path, const std::string& name, int64_t record, int64_t cap, double* out);

}  // namespace ncio
