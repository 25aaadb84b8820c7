/*
 * broccoli_nifti.h -- NIfTI-1 volumes for the command-line tools and hosts
 * that read images from disk (libbroccoli_b200, C ABI, no CUDA involved).
 *
 * Replaces the nifticlib reading and writing of the reference's tools
 * (code/Bash_Wrapper/MotionCorrection.cpp:284-530,
 * code/Bash_Wrapper/HelpFunctions.cpp:325-400):
 *   - reading: a single-file NIfTI-1 image (.nii, or .nii.gz through zlib),
 *     either byte order; voxels of type UINT8, INT8, INT16, UINT16, INT32,
 *     UINT32, FLOAT32 or FLOAT64 are converted to float by a plain cast, as
 *     the reference's tools do (scl_slope / scl_inter are not applied).
 *   - writing: FLOAT32 voxels under a copy of a template header (the input
 *     image's), with the dimensions, datatype, bitpix, vox_offset (352),
 *     cal_min and cal_max set, as WriteNifti does; .gz paths are compressed.
 * Separate .hdr/.img pairs are not read (BRC_ERR_UNSUPPORTED).
 */
#ifndef BROCCOLI_NIFTI_H
#define BROCCOLI_NIFTI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  unsigned char header[348]; /* the header, in this machine's byte order     */
  int dim[8];                /* dim[0] = number of dimensions, then sizes     */
  float pixdim[8];           /* pixdim[1..3] = voxel sizes (mm)               */
  int datatype;              /* the file's NIfTI datatype code                */
  float* data;               /* dim[1] x dim[2] x ... floats, x fastest       */
} brc_nifti;

/* Reads path into *img (img->data allocated by the library; release with
 * brc_nifti_free).  Returns BRC_OK, BRC_ERR_INVALID (not a readable NIfTI-1
 * single file), BRC_ERR_UNSUPPORTED (datatype, or a .hdr/.img pair) or
 * BRC_ERR_NOMEM; brc_nifti_error() then says why. */
int brc_nifti_read(const char* path, brc_nifti* img);

/* Writes nx x ny x nz x nt floats (x fastest) to path as FLOAT32 under the
 * header of `like` (NULL: a minimal header with voxel sizes 1).  A path
 * ending in ".gz" is compressed. */
int brc_nifti_write(const char* path, const brc_nifti* like, const float* data, int nx, int ny, int nz, int nt);

/* Releases img->data (and sets it to NULL). */
void brc_nifti_free(brc_nifti* img);

/* Message of the last failed brc_nifti_* call of this thread. */
const char* brc_nifti_error(void);

#ifdef __cplusplus
}
#endif

#endif
