/* Parcel and field files in the layout of the reference's netCDF output
 * (parcel_netcdf.f90:100-200 and 600-700, field_netcdf.f90:100-250 and
 * 306-389, netcdf_writer.f90:374-600), written in the netCDF classic format:
 * CDF-2, or CDF-5 when a variable exceeds 4 GiB.  The netCDF library reads
 * both, so the reference restarts from these files (utils.f90:200-240,
 * restart_file / field_file); its own netCDF-4 (HDF5) files are not parsed
 * here.  Classic files have no groups: the zeta boundary flags that the
 * reference keeps in its "parameters" group (parameters.f90:220-265) are
 * global attributes of the same names.
 *
 * Parcel files: global attributes file_type = "parcels", ncells, extent,
 * origin; one record (t); variables x_position, y_position, z_position,
 * B11, B12, B13, B22, B23, volume, x_vorticity, y_vorticity, z_vorticity,
 * buoyancy, humidity over (t, n_parcels).  Field files: file_type =
 * "fields", dimensions x, y, z (nz+1 points), t; variables over (t, z, y, x)
 * without halo rows.  All functions return 0 or an EPIC_ERR_* code.  The
 * environment variable EPIC_NC_VERSION=5 makes the writers use CDF-5 for
 * every file. */
#ifndef EPIC_NC_H
#define EPIC_NC_H

#include <stdint.h>

#include "epic_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Host arrays only (no device). */
const char* epic_nc_last_error(void);   /* message of the last failed epic_nc_* call of this thread */
/* What a file holds: file_type ("parcels" / "fields", NUL-terminated, at most
 * 15 characters), the box, the number of parcels (parcel files), the number
 * of records and the time of the last one; zeta_flags = -1 when absent. */
int epic_nc_info(const char* path, char file_type[16], int32_t ncells[3], double origin[3], double extent[3],
                 int64_t* n_parcels, int64_t* n_steps, double* t, int32_t zeta_flags[2]);
/* Arrays as epic_gpu_set_parcels: pos, vor (3,n); B (5,n); vol, buoy, hum (n)
 * (hum may be NULL: zero). */
int epic_nc_write_parcels(const char* path, const int32_t ncells[3], const double origin[3],
                          const double extent[3], const int32_t zeta_flags[2], double t, int64_t n,
                          const double* pos, const double* vor, const double* B, const double* vol,
                          const double* buoy, const double* hum);
/* *n = parcels in the file; fails with EPIC_ERR_ARG if cap < *n. */
int epic_nc_read_parcels(const char* path, int64_t cap, int64_t* n, double* pos, double* vor, double* B,
                         double* vol, double* buoy, double* hum);
/* Record step (0-based; -1 the last) of a field variable into the layout of
 * epic_gpu_set_field for the given box, rows 0 .. nz (the other rows are left
 * as they are).  EPIC_ERR_IO if the file lacks it. */
int epic_nc_read_field(const char* path, const char* name, int64_t step, const int32_t ncells[3],
                       const double origin[3], const double extent[3], double* out);

/* Record `record` (0-based; ignored for a fixed-size variable) of any numeric
 * variable, converted to double in C order; *n = its element count
 * (out NULL: the count only; EPIC_ERR_IO if it exceeds cap). */
int epic_nc_read_variable(const char* path, const char* name, int64_t record, int64_t cap, int64_t* n,
                          double* out);
/* A field file of nfields FP64 fields (names[k], units[k] or NULL for "1"),
 * each in the layout of epic_gpu_set_field (rows 0 .. nz are written), e.g.
 * the vorticity, buoyancy and humidity of an initial state. */
int epic_nc_write_field_file(const char* path, const int32_t ncells[3], const double origin[3],
                             const double extent[3], const int32_t zeta_flags[2], double t, int nfields,
                             const char* const* names, const char* const* units, const double* const* data);

/* Through a context. */
/* write_netcdf_parcels (parcel_netcdf.f90:206-350): the context's parcels at time t. */
int epic_gpu_write_parcels_nc(epic_ctx* ctx, const char* path, double t);
/* read_netcdf_parcels + setup_restart (parcel_netcdf.f90:400-560, utils.f90:144-160):
 * the file's box must be the context's; *t = the file's time (may be NULL).
 * Call init_correction after, as the reference does. */
int epic_gpu_read_parcels_nc(epic_ctx* ctx, const char* path, double* t);
/* write_netcdf_fields (field_netcdf.f90:180-260): velocity, vorticity
 * tendency, parcel counts, vorticity, buoyancy, dry buoyancy, liquid-water
 * content, humidity and volume as they are on the device at time t. */
int epic_gpu_write_fields_nc(epic_ctx* ctx, const char* path, double t);
/* read_netcdf_fields (last record) + init_parcels_from_grids +
 * set_zeta_boundary_flag (utils.f90:223-234): epic_gpu_init_from_grids on
 * the file's x/y/z_vorticity, buoyancy and humidity (absent ones zero). */
int epic_gpu_init_from_field_file(epic_ctx* ctx, const char* path, int32_t zeta_flags[2]);

#ifdef __cplusplus
}
#endif

#endif
