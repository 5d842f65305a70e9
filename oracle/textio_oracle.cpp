// ORACLE — test infrastructure only.  Only tests/ and bench.py's CPU-baseline
// leg load this; the shipped library never links or calls it.
//
// CPU restatement of the reference's INC / GSLIB property file readers and
// writers with the C library's stdio, as the reference does them:
//   read_prop_name            read_inc_file.cpp:8-50
//   load_floats_into_vector   read_inc_file.cpp:52-86
//   read_bytes                read_inc_file.cpp:88-122
//   read_inc_file_float/byte  read_inc_file.cpp:124-178
//   byte remap after reading  api.cpp:69-99
//   writers                   property_writer.cpp:18-147
// Parity of the restatement is pinned by comparing its files and arrays
// with the reference's own entry points compiled by oracle/build_ref.sh.
//
// Where the reference never returns the restatement raises an error instead,
// as the GPU reader does: a '\n' as the first byte of the file is skipped as
// a blank line (the reference retries it forever), the end of the file right
// after a 1023-byte piece of a skipped line ends the name search, and a
// file that runs out of values while the last token read is a comment, or
// before any token was read, ends with "Unexpected end of data.".
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct OracleError {
    std::string msg;
};

bool ascii_letter(unsigned char c) { return (unsigned)((c | 32) - 'a') < 26u; }

void read_prop_name(FILE *f) {
    char line[1024];
    for (;;) {
        line[0] = 0;
        int r = fscanf(f, "%1023[^\n]\n", line);
        size_t n = strlen(line);
        if (r == 0 || n == 0) {
            if (feof(f)) throw OracleError{"read_prop_name: Property name not found."};
            fgetc(f);  // the reference retries this '\n' forever
            continue;
        }
        const bool name = ascii_letter((unsigned char)line[0]);
        while (n == 1023) {
            r = fscanf(f, "%1023[^\n]\n", line);
            if (r == 0) break;
            if (r == EOF) throw OracleError{"read_prop_name: Property name not found."};
            n = strlen(line);
        }
        if (name) return;
    }
}

// The token loop shared by the float and byte readers; `take` converts one
// token or returns false.
template <typename Take>
void read_tokens(FILE *f, long long size, const char *where, Take take) {
    char buffer[256];
    bool have = false;
    for (long long i = 0; i < size;) {
        const int r = fscanf(f, "%255s", buffer);
        if (ferror(f)) throw OracleError{std::string(where) + ": Error reading file."};
        if (r == EOF) {
            // the reference converts the last token read again
            if (!have) throw OracleError{std::string(where) + ": Unexpected end of data."};
        } else {
            have = true;
        }
        const size_t len = strlen(buffer);
        if (len >= 2 && buffer[0] == '-' && buffer[1] == '-') {
            if (r == EOF) throw OracleError{std::string(where) + ": Unexpected end of data."};
            if (fscanf(f, "%*[^\n]") < 0) {
            }
            continue;
        }
        if (len >= 1 && buffer[0] == '/') throw OracleError{std::string(where) + ": Unexpected end of data."};
        if (!take(i, buffer))
            throw OracleError{std::string("load_floats_into_vector: Error parsing '") + buffer + "' string."};
        ++i;
    }
}

void write_float_line(FILE *f, float v) { fprintf(f, "%E\n", (double)v); }
void write_byte_line(FILE *f, unsigned char v) { fprintf(f, "%d\n", (int)(char)v); }

void fail(char *err, int err_len, const std::string &m) {
    if (err && err_len > 0) {
        strncpy(err, m.c_str(), (size_t)err_len - 1);
        err[err_len - 1] = 0;
    }
}

}  // namespace

extern "C" {

// hpgl_read_inc_file_float / hpgl_read_inc_file_byte.  Returns 0, or 1 with
// the reference's message in err.  On error the values stored before the
// failing token stay in the buffers, as in the reference.
int oracle_read_inc(const char *filename, int is_byte, float undef_f, int undef_i, long long size, float *data_f,
                    unsigned char *data_b, unsigned char *mask, const unsigned char *values, int values_count,
                    char *err, int err_len) {
    FILE *f = fopen(filename, "r");
    if (!f) {
        fail(err, err_len, std::string("read_inc_file_float: Error opening file:") + filename + ".");
        return 1;
    }
    try {
        read_prop_name(f);
        if (is_byte) {
            read_tokens(f, size, "read_bytes", [&](long long i, const char *tok) {
                int v;
                if (sscanf(tok, "%d", &v) != 1) return false;
                data_b[i] = (unsigned char)v;
                mask[i] = v == undef_i ? 0 : 1;
                return true;
            });
            for (long long i = 0; i < size; ++i) {
                if (!mask[i]) continue;
                for (int j = 0; j < values_count; ++j)
                    if (data_b[i] == values[j]) {
                        data_b[i] = (unsigned char)j;
                        break;
                    }
            }
        } else {
            read_tokens(f, size, "load_floats_into_vector", [&](long long i, const char *tok) {
                float v;
                if (sscanf(tok, "%f", &v) != 1) return false;
                data_f[i] = v;
                return true;
            });
            for (long long i = 0; i < size; ++i) mask[i] = data_f[i] == undef_f ? 0 : 1;
        }
    } catch (const OracleError &e) {
        fclose(f);
        fail(err, err_len, e.msg);
        return 1;
    }
    fclose(f);
    return 0;
}

// Value tokens before the first '/' outside a comment, or before the end of
// the file; -1 with a message on error.
long long oracle_inc_count(const char *filename, char *err, int err_len) {
    FILE *f = fopen(filename, "r");
    if (!f) {
        fail(err, err_len, std::string("read_inc_file_float: Error opening file:") + filename + ".");
        return -1;
    }
    long long n = 0;
    try {
        read_prop_name(f);
        char buffer[256];
        while (fscanf(f, "%255s", buffer) == 1) {
            const size_t len = strlen(buffer);
            if (len >= 2 && buffer[0] == '-' && buffer[1] == '-') {
                if (fscanf(f, "%*[^\n]") < 0) {
                }
                continue;
            }
            if (buffer[0] == '/') break;
            ++n;
        }
    } catch (const OracleError &e) {
        fclose(f);
        fail(err, err_len, e.msg);
        return -1;
    }
    fclose(f);
    return n;
}

// The four writers: format 0 = INC, 1 = GSLIB.  remap: the byte table
// (init_remap_table's result).
int oracle_write_prop(int format, int is_byte, const char *filename, const char *name, const float *data_f,
                      const unsigned char *data_b, const unsigned char *mask, long long size, float undef_f,
                      unsigned char undef_b, const unsigned char *remap, int remap_count, char *err, int err_len) {
    if (is_byte)
        for (long long i = 0; i < size; ++i)
            if (mask[i] && data_b[i] >= remap_count) {
                fail(err, err_len, "an informed value is outside the table of indicator values");
                return 1;
            }
    FILE *f = fopen(filename, "w+");
    if (!f) {
        fail(err, err_len, std::string("open_file_checked: Can't open file '") + filename + "'.");
        return 1;
    }
    if (format == 1) fprintf(f, "HPGL saved GSLIB file\n%d\n", 1);
    fprintf(f, "%s\n", name);
    for (long long i = 0; i < size; ++i) {
        if (is_byte) write_byte_line(f, mask[i] ? remap[data_b[i]] : undef_b);
        else write_float_line(f, mask[i] ? data_f[i] : undef_f);
    }
    if (format == 0) fprintf(f, "/\n");
    fclose(f);
    return 0;
}
}
