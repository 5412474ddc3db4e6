/* Minimal HDF5 input/output for the reference's data formats, without
 * libhdf5 (host code in libraptr_b200.so).
 *
 * Replaces, for the two layouts raptr's tools exchange (README.md "Data
 * Formats"):
 *   H5Reader (src/H5Reader.hpp:34-102) and readHDF5_MeasVct /
 *   readHDF5_MeasList / readHDF5_Density (src/wrappers.hpp:330-410,471-482):
 *     raptr_h5_dataset_info, raptr_h5_read_f32, raptr_h5_read_density_grid;
 *   H5DensityWriter<TGrid>::write (src/H5DensityWriter.hpp:97-232) and
 *   writeHDF5_Density (src/wrappers.hpp:417-422): raptr_h5_write_density;
 *   the measurement files the reference reads: raptr_h5_write_measurement.
 *
 * Files are written in the earliest HDF5 form (superblock 0, version-1
 * object headers, symbol-table root group, contiguous little-endian
 * datasets); the reader reads that form (including libhdf5's continuation
 * blocks) and reports other layouts as unsupported.  The C++ functions with
 * the reference's names are in raptr_b200.hpp. */
#ifndef RAPTR_B200_H5_H
#define RAPTR_B200_H5_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RAPTR_H5_OK 0
#define RAPTR_H5_INVALID 1     /* bad argument or buffer too small            */
#define RAPTR_H5_IO 2          /* the file cannot be opened / read / written  */
#define RAPTR_H5_FORMAT 3      /* not HDF5 or a structure is damaged          */
#define RAPTR_H5_UNSUPPORTED 4 /* a valid HDF5 form this reader does not read */
#define RAPTR_H5_NOT_FOUND 5   /* no dataset of that name in the root group   */

const char* raptr_h5_last_error(void);

/* Measurement file: dataset "messung", float32, dims (angles, z0, y0, z1,
 * y1), data in channel id order. */
int raptr_h5_write_measurement(const char* path, const float* data, const int64_t dims[5]);
/* Density file: dataset "density", float32, dims (nx, ny, nz) with x
 * slowest, attributes xmin/xmax/ymin/ymax/zmin/zmax (float) and
 * xnbin/ynbin/znbin (int32). */
int raptr_h5_write_density(const char* path, const float* data, const int32_t n[3], const float lo[3],
                           const float hi[3]);
/* Rank and dims of a dataset of the root group. */
int raptr_h5_dataset_info(const char* path, const char* name, int32_t* rank, int64_t dims[8]);
/* Reads a dataset (float32, float64 or int32) as float; *count = elements.
 * With out == NULL only *count is set. */
int raptr_h5_read_f32(const char* path, const char* name, float* out, int64_t capacity, int64_t* count);
/* Grid attributes of a density file. */
int raptr_h5_read_density_grid(const char* path, int32_t n[3], float lo[3], float hi[3]);

#ifdef __cplusplus
}
#endif

#endif /* RAPTR_B200_H5_H */
