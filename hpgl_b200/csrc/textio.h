// Eclipse INC / GSLIB property files on the GPU (textio.cu).
#pragma once
#include <string>

namespace hpgl_b200 {

// Host-side timings of one call, milliseconds.
struct TextIoTiming {
    double ms_file = 0;    // reading or writing the file (host)
    double ms_h2d = 0;     // host -> device copies
    double ms_device = 0;  // kernels (CUDA events)
    double ms_d2h = 0;     // device -> host copies
    double ms_total = 0;
    long long bytes = 0;   // file size
    long long tokens = 0;  // whitespace-separated tokens of the data section
};

// Reads `size` values of an INC file (read_inc_file.cpp:128-178): the
// property name line, then whitespace-separated values, "--" comments to the
// end of the line, "/" ends the data.  With is_byte the values are integers
// (read_bytes), stored as bytes with mask = (value != undefined), and then
// remapped through `values` (api.cpp:69-99); else floats with mask =
// (value != undefined).  Errors throw HpglError with the reference's
// messages.
void inc_read(const char *filename, bool is_byte, float undefined_f, int undefined_i, long long size,
              float *data_f, unsigned char *data_b, unsigned char *mask, const unsigned char *values,
              int values_count, TextIoTiming *timing);

// Number of values an INC file holds: value tokens before the first '/'
// that is not in a comment, or before the end of the file.
long long inc_count(const char *filename, bool is_byte, TextIoTiming *timing);

// Writes a property (property_writer.cpp:18-214): format 0 = INC (name
// line, one value per line, "/" line), 1 = GSLIB ("HPGL saved GSLIB file",
// "1", name line, one value per line).  Floats as "%E" of the value widened
// to double; bytes as "%d" of (char)remap[value]; uninformed cells as the
// undefined value.
void prop_write(int format, bool is_byte, const char *filename, const char *name, const float *data_f,
                const unsigned char *data_b, const unsigned char *mask, long long size, float undefined_f,
                unsigned char undefined_b, const unsigned char *remap, int remap_count, TextIoTiming *timing);

// Timing of the last inc_read / inc_count / prop_write / variogram call.
TextIoTiming last_io_timing();
void set_last_io_timing(const TextIoTiming &t);

}  // namespace hpgl_b200
