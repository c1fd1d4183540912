/*
 * vct_io.h -- the reference's input-txt and raw-file formats (host side of
 * the drop-in executables vct_mbfpa and vct_fbp).
 *
 * The txt format is positional: 6 header lines, then for every field two
 * skipped lines and one value line (MB/projectionDataTOMO.cpp:17-64).
 */
#ifndef VCT_IO_H
#define VCT_IO_H

#include <stddef.h>
#include <stdint.h>

#include "vct.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The 31 fields of the MBFPA input txt, MB/projectionDataTOMO.h:2-68 and
 * MB/projectionDataTOMO.cpp:83-121, plus the derived values of :126-134 and
 * :332-333. */
typedef struct vct_mb_config {
  char in_pr_class[16];          /* "PR" or "IN" */
  int prior_image_onoff;
  int proj_width;                /* projImgWidth */
  int proj_height;               /* projImgHeight after derivation */
  char proj_data_type[16];
  int proj_file_offset;
  char proj_file[256];
  char air_scan_file[256];
  double gantry_rotation_period;
  double data_sampling_rate;     /* after the >= 200 Hz thinning */
  double data_sampling_rate_orig;
  double start_view_angle;
  double couch_speed;
  double start_couch_position;
  int recon_size;
  double recon_pix_size;
  char recon_tgt_class[16];
  double recon_offset;
  double recon_step;
  int recon_slices;
  int xfactor;
  char recon_data_file[256];     /* prior image */
  int fbp_slice;
  double x_reg, y_reg, z_reg;    /* z_reg after the ScanListZvalue update (:109) */
  double scan_list_z;
  int osemset;
  double total_variation, prior_const, markov_const;
  double gradient_decent_const;
  int num_ite;
  int sino_fact;
  char spectrum_file[256];
  double photon_noise;
  int total_proj_number;         /* (int)(txt height/(period*rate_orig)) */
} vct_mb_config;

/* The 21 fields of the FBP input txt, FBP/projectionDataTOMO.cpp:70-96. */
typedef struct vct_fbp_config {
  char in_pr_class[16];
  int filter;                    /* 1 Ram-Lak, 2 Shepp-Logan */
  int proj_width;
  int proj_height;               /* (int)(period*rate) */
  char proj_data_type[16];
  int proj_file_offset;
  char proj_file[256];
  char air_scan_file[256];
  double gantry_rotation_period;
  double data_sampling_rate;
  double start_view_angle;
  double couch_speed;
  double start_couch_position;
  int recon_size;
  double recon_pix_size;
  char recon_tgt_class[16];
  double recon_offset;
  double recon_step;
  int recon_slices;
  int xfactor;
  char output_file[256];         /* reconDataFilename: the output image */
  int total_proj_number;
} vct_fbp_config;

/* Returns VCT_OK, or VCT_E_IO when the file cannot be opened (the reference
 * prints "info file: ... not found" and exits). */
int vct_load_mb_config(const char* path, vct_mb_config* cfg);
int vct_load_fbp_config(const char* path, vct_fbp_config* cfg);

/* Geometry for a parsed config: physParamsTOMO.h defaults + txt fields. */
void vct_mb_geometry(const vct_mb_config* cfg, vct_geometry* g);
void vct_fbp_geometry(const vct_fbp_config* cfg, vct_geometry* g);

/* Reads exactly `bytes` bytes at `offset`; VCT_E_IO on a missing or short
 * file.  *got (optional) receives the byte count actually read. */
int vct_read_raw(const char* path, long offset, void* buf, size_t bytes, size_t* got);
int vct_write_raw(const char* path, const void* buf, size_t bytes);

/* ------------------------------------------------- measured-data ingestion
 * The raw detector layout of a measured sinogram and its air scan: the
 * NumberOfChannels, NumberOfSkips, AirScn_Sinogram_Height,
 * AirScn_Sinogram_Number, Start_Channel and End_Channel constants of
 * MB/physParamsTOMO.h:32-65 as runtime fields. */
typedef struct vct_raw_layout {
  int raw_channels;   /* floats per raw detector row (609) */
  int skip_channels;  /* raw channels before the first used one (27) */
  int air_rows;       /* rows per air-scan block and per PR rotation (800) */
  int air_blocks;     /* air-scan blocks averaged after the first, unused one (5) */
  int start_channel;  /* raw-channel window of the IN-mode maximum check */
  int end_channel;    /*   [start_channel, end_channel): 0 and 609 */
} vct_raw_layout;
void vct_raw_layout_default(vct_raw_layout* layout);

/* loadProjectionData, MB/projectionDataTOMO.cpp:324-508: reads
 * cfg->air_scan_file and cfg->proj_file and writes the normalised volume
 * [cfg->total_proj_number][cfg->proj_height][cfg->proj_width] and its mask
 * (1 = usable).  The air scan's first block is skipped and the next
 * air_blocks are averaged in float, block by block.
 *   PR (cfg->in_pr_class "PR"): each rotation is an [air_rows][raw_channels]
 *      plane; volume = plane / air mean over channels skip_channels.., rows
 *      thinned by cfg->sino_fact; mask 1.
 *   IN: rows of raw_channels floats per view (5 per view when
 *      cfg->data_sampling_rate_orig >= 200, the first used); volume =
 *      row / (2 * air mean of air row 0), values below 0.1 set to 0 with
 *      mask 0.  As in the reference's loop, only view 0 of each rotation
 *      reads the file's row; views >= 1 read rows of its buffer that no read
 *      fills, so they are 0 (or NaN where the air mean is 0).
 * Files are read with the reference's byte counts into buffers that persist
 * between reads: a short file repeats the previous read's tail.  Returns
 * VCT_E_IO when a file is missing (the reference then keeps a zero volume),
 * VCT_E_RANGE when an IN-mode value in [start_channel, end_channel) exceeds 1
 * (the reference prints it and stops; *max_value = that value),
 * VCT_E_UNSUPPORTED for layouts that would take the reference past its own
 * buffers (PR: skip_channels + width > raw_channels or kept air rows !=
 * proj_height; IN: rows read past one air block).  *rotations receives the
 * rotations read, *max_value the IN-mode maximum in the window (0 for PR).
 * The normalisation runs on `device`; _dev writes device buffers on stream
 * and returns after it has finished with its host copies. */
int vct_load_measured(const vct_mb_config* cfg, const vct_raw_layout* layout, int device, float* volume,
                      unsigned char* mask, int* rotations, double* max_value);
int vct_load_measured_dev(const vct_mb_config* cfg, const vct_raw_layout* layout, float* d_volume,
                          unsigned char* d_mask, int* rotations, double* max_value, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VCT_IO_H */
