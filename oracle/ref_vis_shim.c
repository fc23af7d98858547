/*
 * Visibility-file oracle (TEST INFRASTRUCTURE ONLY): the tag sequence of the
 * reference's .vis header and block writers, restated here because their
 * sources need a header that the reference's build system generates
 * (oskar_version.h), written through the reference's own binary-format
 * library (binary/src/*.c, compiled from its sources by `make -C oracle
 * ref`: chunk tags, CRC-32C and file header are the reference's code).
 * Nothing in the product links it.
 *
 * orcvis_create follows oskar_vis_header_write
 * (vis/src/oskar_vis_header_write.c:20-253) with the header fields that
 * oskar_vis_header_create and the simulator set
 * (vis/src/oskar_vis_header_create.c:20-129,
 * interferometer/src/oskar_interferometer_check_init.c:128-266);
 * orcvis_write_block follows oskar_vis_block_write
 * (vis/src/oskar_vis_block_write.c:16-70).
 */
#include <stdlib.h>
#include <string.h>

#include "binary/oskar_binary.h"

#define GRP_HDR 11 /* OSKAR_TAG_GROUP_VIS_HEADER */
#define GRP_BLK 12 /* OSKAR_TAG_GROUP_VIS_BLOCK */

static size_t orc_elem(int type)
{
    size_t s = (type & 1) ? 1 : (type & 2) ? sizeof(int) : (type & 4) ?
            sizeof(float) : sizeof(double);
    if (type & 0x20) s *= 2;
    if (type & 0x40) s *= 4;
    return s;
}

typedef struct
{
    oskar_Binary* h;
    int amp_type, coord_type, num_stations, write_auto, write_cross;
    int status;
} orcvis;

void* orcvis_create(const char* filename, int amp_type, int coord_precision,
        int max_times_per_block, int num_times_total,
        int max_channels_per_block, int num_channels_total, int num_stations,
        int write_autocorr, int write_crosscorr, int casa,
        double freq_start_hz, double freq_inc_hz, double bandwidth_hz,
        double time_start_mjd, double time_inc_sec, double time_average_sec,
        int pc_type, double pc_lon_deg, double pc_lat_deg, double lon_deg,
        double lat_deg, double alt_m, const void* sx, const void* sy,
        const void* sz, const double* diameter,
        const char* const* names, const int* num_elements, const void* ex,
        const void* ey, const void* ez, const double* feed_angles,
        const char* telescope_path, const char* settings,
        const char* date_time, const char* version, const char* cwd,
        const char* username)
{
    orcvis* v = (orcvis*) calloc(1, sizeof(orcvis));
    int* st = &v->status;
    int i = 0, tags = 1, d = 0, f = 0;
    size_t total = 0, off = 0;
    const size_t cs = orc_elem(coord_precision);
    double pc[2];
    double* diam = (double*) calloc((size_t) num_stations + 1,
            sizeof(double));
    v->amp_type = amp_type;
    v->coord_type = coord_precision;
    v->num_stations = num_stations;
    v->write_auto = write_autocorr;
    v->write_cross = write_crosscorr;
    v->h = oskar_binary_create(filename, 'w', st);
    /* metadata (oskar_vis_header_write.c:40-87) */
    oskar_binary_write(v->h, OSKAR_CHAR, OSKAR_TAG_GROUP_METADATA,
            OSKAR_TAG_METADATA_DATE_TIME_STRING, 0, 1 + strlen(date_time),
            date_time, st);
    oskar_binary_write(v->h, OSKAR_CHAR, OSKAR_TAG_GROUP_METADATA,
            OSKAR_TAG_METADATA_OSKAR_VERSION_STRING, 0, 1 + strlen(version),
            version, st);
    if (cwd)
        oskar_binary_write(v->h, OSKAR_CHAR, OSKAR_TAG_GROUP_METADATA,
                OSKAR_TAG_METADATA_CWD, 0, 1 + strlen(cwd), cwd, st);
    if (username && strlen(username) > 0)
        oskar_binary_write(v->h, OSKAR_CHAR, OSKAR_TAG_GROUP_METADATA,
                OSKAR_TAG_METADATA_USERNAME, 0, 1 + strlen(username),
                username, st);
    if (settings && strlen(settings) > 0)
        oskar_binary_write(v->h, OSKAR_CHAR, OSKAR_TAG_GROUP_SETTINGS,
                OSKAR_TAG_SETTINGS, 0, strlen(settings), settings, st);
    /* header fields (oskar_vis_header_write.c:89-199) */
    oskar_binary_write(v->h, OSKAR_CHAR, GRP_HDR, 1, 0,
            telescope_path ? strlen(telescope_path) + 1 : 0, telescope_path,
            st);
    if (write_crosscorr) tags += 4;
    if (write_autocorr) tags += 1;
    if (max_times_per_block <= 0) max_times_per_block = num_times_total;
    if (max_channels_per_block <= 0)
        max_channels_per_block = num_channels_total;
    oskar_binary_write_int(v->h, GRP_HDR, 2, 0, tags, st);
    oskar_binary_write_int(v->h, GRP_HDR, 3, 0, write_autocorr, st);
    oskar_binary_write_int(v->h, GRP_HDR, 4, 0, write_crosscorr, st);
    oskar_binary_write_int(v->h, GRP_HDR, 5, 0, amp_type, st);
    oskar_binary_write_int(v->h, GRP_HDR, 6, 0, coord_precision, st);
    oskar_binary_write_int(v->h, GRP_HDR, 7, 0, max_times_per_block, st);
    oskar_binary_write_int(v->h, GRP_HDR, 8, 0, num_times_total, st);
    oskar_binary_write_int(v->h, GRP_HDR, 9, 0, max_channels_per_block, st);
    oskar_binary_write_int(v->h, GRP_HDR, 10, 0, num_channels_total, st);
    oskar_binary_write_int(v->h, GRP_HDR, 11, 0, num_stations, st);
    oskar_binary_write_int(v->h, GRP_HDR, 12, 0,
            (amp_type & 0x40) ? 10 : 1, st);
    oskar_binary_write_int(v->h, GRP_HDR, 13, 0, casa, st);
    oskar_binary_write_int(v->h, GRP_HDR, 21, 0, pc_type, st);
    pc[0] = pc_lon_deg;
    pc[1] = pc_lat_deg;
    oskar_binary_write(v->h, OSKAR_DOUBLE, GRP_HDR, 22, 0, sizeof(pc), pc,
            st);
    oskar_binary_write_double(v->h, GRP_HDR, 23, 0, freq_start_hz, st);
    oskar_binary_write_double(v->h, GRP_HDR, 24, 0, freq_inc_hz, st);
    oskar_binary_write_double(v->h, GRP_HDR, 25, 0, bandwidth_hz, st);
    oskar_binary_write_double(v->h, GRP_HDR, 26, 0, time_start_mjd, st);
    oskar_binary_write_double(v->h, GRP_HDR, 27, 0, time_inc_sec, st);
    oskar_binary_write_double(v->h, GRP_HDR, 28, 0, time_average_sec, st);
    oskar_binary_write_double(v->h, GRP_HDR, 29, 0, lon_deg, st);
    oskar_binary_write_double(v->h, GRP_HDR, 30, 0, lat_deg, st);
    oskar_binary_write_double(v->h, GRP_HDR, 31, 0, alt_m, st);
    /* stations and elements (oskar_vis_header_write.c:201-219) */
    oskar_binary_write(v->h, (unsigned char) coord_precision, GRP_HDR, 32,
            0, cs * num_stations, sx, st);
    oskar_binary_write(v->h, (unsigned char) coord_precision, GRP_HDR, 33,
            0, cs * num_stations, sy, st);
    oskar_binary_write(v->h, (unsigned char) coord_precision, GRP_HDR, 34,
            0, cs * num_stations, sz, st);
    for (i = 0; i < num_stations; ++i)
        total += num_elements ? (size_t) num_elements[i] : 0;
    for (i = 0, off = 0; i < num_stations; ++i)
    {
        const size_t n = num_elements ? (size_t) num_elements[i] : 0;
        const int have = n && ex && ey && ez;
        oskar_binary_write(v->h, (unsigned char) coord_precision, GRP_HDR,
                35, i, have ? cs * n : 0,
                have ? (const char*) ex + cs * off : 0, st);
        oskar_binary_write(v->h, (unsigned char) coord_precision, GRP_HDR,
                36, i, have ? cs * n : 0,
                have ? (const char*) ey + cs * off : 0, st);
        oskar_binary_write(v->h, (unsigned char) coord_precision, GRP_HDR,
                37, i, have ? cs * n : 0,
                have ? (const char*) ez + cs * off : 0, st);
        off += n;
    }
    /* names and diameters (oskar_vis_header_write.c:221-232); an unset
     * name is the one zero byte oskar_vis_header_create allocates */
    for (i = 0; i < num_stations; ++i)
    {
        const char* s = (names && names[i]) ? names[i] : "";
        oskar_binary_write(v->h, OSKAR_CHAR, GRP_HDR, 41, i, strlen(s) + 1,
                s, st);
    }
    if (diameter)
        memcpy(diam, diameter, sizeof(double) * num_stations);
    oskar_binary_write(v->h, OSKAR_DOUBLE, GRP_HDR, 42, 0,
            sizeof(double) * num_stations, diam, st);
    free(diam);
    /* feed angles: per station X_A, Y_A, X_B, Y_B, X_C, Y_C
     * (oskar_vis_header_write.c:234-251) */
    for (i = 0, off = 0; i < num_stations; ++i)
    {
        const size_t n = num_elements ? (size_t) num_elements[i] : 0;
        for (d = 0; d < 3; ++d)
            for (f = 0; f < 2; ++f)
            {
                const int have = n && feed_angles;
                oskar_binary_write(v->h, OSKAR_DOUBLE, GRP_HDR,
                        (unsigned char) (43 + 2 * d + f), i,
                        have ? sizeof(double) * n : 0,
                        have ? feed_angles + (3 * f + d) * total + off : 0,
                        st);
            }
        off += n;
    }
    return v;
}

int orcvis_write_block(void* p, int block_index, int start_time,
        int start_channel, int num_times, int num_channels,
        const void* cross, const void* autos, const void* su,
        const void* sv, const void* sw)
{
    orcvis* v = (orcvis*) p;
    int* st = &v->status;
    const int n = v->num_stations;
    const int nbl = v->write_cross ? n * (n - 1) / 2 : 0;
    const size_t es = orc_elem(v->amp_type);
    const size_t tc = (size_t) num_times * num_channels;
    int dims[6];
    dims[0] = start_time;
    dims[1] = start_channel;
    dims[2] = num_times;
    dims[3] = num_channels;
    dims[4] = nbl;
    dims[5] = n;
    oskar_binary_write(v->h, OSKAR_INT, GRP_BLK, 1, block_index,
            sizeof(dims), dims, st);
    if (v->write_auto && tc * n > 0)
        oskar_binary_write(v->h, (unsigned char) v->amp_type, GRP_BLK, 2,
                block_index, es * tc * n, autos, st);
    if (v->write_cross && tc * nbl > 0)
    {
        oskar_binary_write(v->h, (unsigned char) v->amp_type, GRP_BLK, 3,
                block_index, es * tc * nbl, cross, st);
        if (su && sv && sw)
        {
            const size_t b = orc_elem(v->coord_type) * num_times * n;
            oskar_binary_write(v->h, (unsigned char) v->coord_type, GRP_BLK,
                    7, block_index, b, su, st);
            oskar_binary_write(v->h, (unsigned char) v->coord_type, GRP_BLK,
                    8, block_index, b, sv, st);
            oskar_binary_write(v->h, (unsigned char) v->coord_type, GRP_BLK,
                    9, block_index, b, sw, st);
        }
    }
    return *st;
}

int orcvis_close(void* p)
{
    orcvis* v = (orcvis*) p;
    const int st = v->status;
    oskar_binary_free(v->h);
    free(v);
    return st;
}

/* Reads one chunk back with the reference's reader (CRC checked); returns
 * the reader's status. */
int orcvis_read(const char* filename, int data_type, int group, int tag,
        int index, size_t bytes, void* data)
{
    int st = 0;
    oskar_Binary* h = oskar_binary_create(filename, 'r', &st);
    if (!st)
        oskar_binary_read(h, (unsigned char) data_type,
                (unsigned char) group, (unsigned char) tag, index, bytes,
                data, &st);
    if (h) oskar_binary_free(h);
    return st;
}

/* Number of chunks the reference's reader indexes in the file. */
int orcvis_num_tags(const char* filename)
{
    int st = 0, n = -1;
    oskar_Binary* h = oskar_binary_create(filename, 'r', &st);
    if (!st) n = oskar_binary_num_tags(h);
    if (h) oskar_binary_free(h);
    return st ? st : n;
}
