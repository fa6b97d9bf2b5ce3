"""ctypes mirrors of the structs declared in include/freect_wfbp.h.

CTGeometry, ReconConfig and GPUPrecompute keep the field order and types of
the reference's applications/fct_wfbp/include/recon_structs.h:6-31, 33-50,
52-67, so a buffer filled by the reference's host code has the same layout.
"""
import ctypes as C

c_size_t = C.c_size_t


class CTGeometry(C.Structure):
    """recon_structs.h:6-31"""
    _fields_ = [
        ("total_number_of_projections", c_size_t),
        ("projections_per_rotation", c_size_t),
        ("detector_pixel_size_col", C.c_float),
        ("detector_pixel_size_row", C.c_float),
        ("num_detector_cols", c_size_t),
        ("num_detector_cols_padded", c_size_t),
        ("num_detector_cols_padded_fft", c_size_t),
        ("num_detector_rows", c_size_t),
        ("num_detector_rows_padded", c_size_t),
        ("detector_central_col", C.c_float),
        ("detector_central_row", C.c_float),
        ("distance_source_to_detector", C.c_float),
        ("distance_source_to_isocenter", C.c_float),
        ("collimated_slice_width", C.c_float),
        ("theta_cone", C.c_float),
        ("acquisition_field_of_view", C.c_float),
        ("z_rot", C.c_float),
        ("anode_angle", C.c_float),
        ("ffs_phi", C.c_bool),
        ("ffs_z", C.c_bool),
        ("ffs_diag", C.c_bool),
    ]


class ReconConfig(C.Structure):
    """recon_structs.h:33-50"""
    _fields_ = [
        ("raw_data_dir", C.c_char * 4096),
        ("output_dir", C.c_char * 4096),
        ("output_file", C.c_char * 255),
        ("start_pos", C.c_float),
        ("end_pos", C.c_float),
        ("recon_fov", C.c_float),
        ("slice_thickness", C.c_float),
        ("slice_pitch", C.c_float),
        ("nx", c_size_t),
        ("ny", c_size_t),
        ("recon_kernel", C.c_int),
        ("x_origin", C.c_float),
        ("y_origin", C.c_float),
        ("tube_angle_offset", C.c_float),
        ("adaptive_filtration_s", C.c_float),
    ]


class GPUPrecompute(C.Structure):
    """recon_structs.h:52-67"""
    _fields_ = [
        ("half_acquisition_fov", C.c_float),
        ("half_acquisition_fov_squared", C.c_float),
        ("projections_per_half_turn", C.c_int),
        ("n_half_turns", C.c_int),
        ("distance_source_to_isocenter_squared", C.c_float),
        ("z_rot_over_2_pi", C.c_float),
        ("recip_distance_source_to_detector", C.c_float),
        ("recip_distance_source_to_isocenter", C.c_float),
        ("tanf_theta_cone", C.c_float),
        ("pixel_scale", C.c_float),
        ("two_pi_over_projections_per_rotation", C.c_float),
        ("n_slices_native", C.c_int),
        ("n_slices_requested", C.c_int),
    ]


class ScanMeta(C.Structure):
    """wfbp_scan_meta: the RawDataSet getters ConfigureCTGeometry reads
    (modules/fct_read/include/fct/RawDataSet.h:90-106)."""
    _fields_ = [
        ("total_num_projections", C.c_int),
        ("projections_per_rotation", C.c_int),
        ("detector_channels", C.c_int),
        ("detector_rows", C.c_int),
        ("detector_transverse_spacing", C.c_float),
        ("detector_axial_spacing", C.c_float),
        ("detector_central_channel", C.c_float),
        ("detector_central_row", C.c_float),
        ("dist_source_to_isocenter", C.c_float),
        ("dist_source_to_detector", C.c_float),
        ("ffs_mode", C.c_int),
        ("anode_angle", C.c_float),
    ]


class Ext(C.Structure):
    """wfbp_ext"""
    _fields_ = [
        ("version", C.c_int),
        ("precision", C.c_int),
        ("filter_window", C.c_int),
        ("filter_c", C.c_float),
        ("filter_a", C.c_float),
        ("user_taps", C.POINTER(C.c_float)),
        ("n_user_taps", C.c_int),
        ("tex_weights", C.c_int),
        ("bp_slab", C.c_int),
        ("filtered_layout", C.c_int),
        ("adjoint_scale_table", C.c_int),
        ("reserved", C.c_int * 5),
    ]


class Dims(C.Structure):
    """wfbp_dims"""
    _fields_ = [
        ("n_views", C.c_int),
        ("n_rows", C.c_int),
        ("n_channels", C.c_int),
        ("n_readings", C.c_int),
        ("raw_rows", C.c_int),
        ("raw_channels", C.c_int),
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("n_slices_native", C.c_int),
        ("n_slices_requested", C.c_int),
        ("precision", C.c_int),
        ("raw_bytes", c_size_t),
        ("rebinned_bytes", c_size_t),
        ("filtered_bytes", c_size_t),
        ("row_scale_bytes", c_size_t),
        ("native_volume_bytes", c_size_t),
        ("volume_bytes", c_size_t),
    ]


class BpConfig(C.Structure):
    """wfbp_bp_config"""
    _fields_ = [("tile_x", C.c_int), ("tile_y", C.c_int), ("cols_per_step", C.c_int), ("consumer_warps", C.c_int),
                ("slab", C.c_int)]

    def key(self):
        return (self.tile_x, self.tile_y, self.cols_per_step, self.consumer_warps, self.slab)


class Ellipsoid(C.Structure):
    """wfbp_ellipsoid"""
    _fields_ = [(n, C.c_double) for n in ("cx", "cy", "cz", "ax", "ay", "az", "phi", "mu")]


class SynthScan(C.Structure):
    """wfbp_synth_scan"""
    _fields_ = [
        ("n_readings", C.c_int),
        ("rows", C.c_int),
        ("channels", C.c_int),
        ("readings_per_rotation", C.c_int),
        ("sid", C.c_double),
        ("sdd", C.c_double),
        ("dcol", C.c_double),
        ("drow", C.c_double),
        ("central_channel", C.c_double),
        ("angle0", C.c_double),
        ("dangle", C.c_double),
        ("z0", C.c_double),
        ("dz", C.c_double),
        ("i0", C.c_double),
        ("seed", C.c_ulonglong),
        ("ffs_mode", C.c_int),
    ]


# enum values (include/freect_wfbp.h)
WFBP_OK = 0
STATUS_NAMES = {0: "WFBP_OK", 1: "WFBP_ERR_INVALID_ARG", 2: "WFBP_ERR_OOM", 3: "WFBP_ERR_CUDA",
                4: "WFBP_ERR_TIMEOUT", 5: "WFBP_ERR_UNSUPPORTED", 6: "WFBP_ERR_STATE"}
PRECISION_FP32 = 0
PRECISION_MIXED = 1
FILTER_REFERENCE = 0
FILTER_SHEPP_LOGAN = 1
FILTER_USER = 2
RECON_KERNEL_RAMLAK = 0
RECON_KERNEL_SHEPP_LOGAN = 1
RECON_KERNEL_HANN = 2
RECON_KERNEL_HAMMING = 3
FFS_NONE, FFS_PHI, FFS_Z, FFS_PHIZ = 0, 1, 2, 3
LAYOUT_REFERENCE = 0
LAYOUT_BACKPROJECTION = 1
EXT_VERSION = 1
