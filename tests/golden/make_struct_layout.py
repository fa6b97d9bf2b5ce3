"""Writes tests/golden/struct_layout.json: sizeof/offsetof of the reference's
CTGeometry, ReconConfig and GPUPrecompute, compiled with g++ from the
reference's own applications/fct_wfbp/include/recon_structs.h.
Run where the reference tree is present: its root is taken from the
FREECT_REFERENCE_ROOT environment variable (default /root/reference) or the
first command-line argument."""
import json
import os
import subprocess
import sys
import tempfile

REF = os.path.join(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FREECT_REFERENCE_ROOT", "/root/reference"),
                   "applications", "fct_wfbp", "include")
FIELDS = {
    "CTGeometry": ["total_number_of_projections", "projections_per_rotation", "detector_pixel_size_col",
                   "detector_pixel_size_row", "num_detector_cols", "num_detector_cols_padded",
                   "num_detector_cols_padded_fft", "num_detector_rows", "num_detector_rows_padded",
                   "detector_central_col", "detector_central_row", "distance_source_to_detector",
                   "distance_source_to_isocenter", "collimated_slice_width", "theta_cone",
                   "acquisition_field_of_view", "z_rot", "anode_angle", "ffs_phi", "ffs_z", "ffs_diag"],
    "ReconConfig": ["raw_data_dir", "output_dir", "output_file", "start_pos", "end_pos", "recon_fov",
                    "slice_thickness", "slice_pitch", "nx", "ny", "recon_kernel", "x_origin", "y_origin",
                    "tube_angle_offset", "adaptive_filtration_s"],
    "GPUPrecompute": ["half_acquisition_fov", "half_acquisition_fov_squared", "projections_per_half_turn",
                      "n_half_turns", "distance_source_to_isocenter_squared", "z_rot_over_2_pi",
                      "recip_distance_source_to_detector", "recip_distance_source_to_isocenter", "tanf_theta_cone",
                      "pixel_scale", "two_pi_over_projections_per_rotation", "n_slices_native",
                      "n_slices_requested"],
}


def layout_program(header_line):
    lines = ["#include <cstdio>", "#include <cstddef>", header_line, "int main(){", 'printf("{");']
    first = True
    for s, fs in FIELDS.items():
        lines.append('printf("%s\\"%s\\": {\\"sizeof\\": %%zu", sizeof(%s));' % ("" if first else ",", s, s))
        for f in fs:
            lines.append('printf(", \\"%s\\": %%zu", offsetof(%s, %s));' % (f, s, f))
        lines.append('printf("}");')
        first = False
    lines += ['printf("}\\n");', "return 0;}"]
    return "\n".join(lines)


def run(header_line, includes, compiler="g++"):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "l.cpp")
        open(src, "w").write(layout_program(header_line))
        exe = os.path.join(d, "l")
        subprocess.check_call([compiler, "-x", "c++", "-O0"] + ["-I" + i for i in includes] + [src, "-o", exe])
        return json.loads(subprocess.check_output([exe]).decode())


if __name__ == "__main__":
    out = run('#include "recon_structs.h"', [REF])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "struct_layout.json")
    json.dump(out, open(path, "w"), indent=1, sort_keys=True)
    print(path, out["CTGeometry"]["sizeof"], out["ReconConfig"]["sizeof"], out["GPUPrecompute"]["sizeof"])
