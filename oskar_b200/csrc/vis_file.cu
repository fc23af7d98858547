// Visibility files in the OSKAR binary format (version 2): the block
// finalisation step of the simulator, writing the visibility header and
// then each block of [time][channel][baseline] visibilities as it is
// finished (oskar/vis/src/oskar_vis_header_write.c:20-253,
// oskar/vis/src/oskar_vis_block_write.c:16-70).
//
// File layout (docs/binary_file/binary_file.rst): a 64-byte file header
// ("OSKARBIN", NUL, format version 2, zeros), then chunks. A chunk is a
// 20-byte tag ('T', 0x40 + version, 'G', payload element size, flags = CRC
// present, data type, group id, tag id, little-endian 4-byte user index,
// little-endian 8-byte block size = payload + 4), the payload, and a
// little-endian CRC-32C (Castagnoli, reflected polynomial 0x82F63B78) of
// tag and payload. The tag sequence and the group / tag identifiers are the
// reference's (the file must read back with its reader); the code is this
// library's own. Host code only: visibilities are written from host memory
// (the block drivers download each block into page-locked host buffers).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace oskb {
namespace {

// Payload type codes (binary_file.rst, "Payload Data Type").
enum { kChar = 0x01, kInt = 0x02, kSingle = 0x04, kDouble = 0x08,
    kComplex = 0x20, kMatrix = 0x40 };

// Tag groups and identifiers (binary_file.rst, "Standard Tag Groups";
// oskar/binary/oskar_binary.h:34-64, oskar/vis/oskar_vis_header.h:27-69,
// oskar/vis/oskar_vis_block.h:27-38).
enum { kGroupMetadata = 1, kGroupSettings = 3, kGroupVisHeader = 11,
    kGroupVisBlock = 12 };
enum { kMetaDateTime = 1, kMetaVersion = 2, kMetaUsername = 3,
    kMetaCwd = 4, kSettingsContents = 2 };
enum
{
    kHdrTelescopePath = 1, kHdrTagsPerBlock = 2, kHdrWriteAuto = 3,
    kHdrWriteCross = 4, kHdrAmpType = 5, kHdrCoordPrecision = 6,
    kHdrMaxTimes = 7, kHdrNumTimes = 8, kHdrMaxChannels = 9,
    kHdrNumChannels = 10, kHdrNumStations = 11, kHdrPolType = 12,
    kHdrCasa = 13, kHdrPhaseCentreType = 21, kHdrPhaseCentreDeg = 22,
    kHdrFreqStart = 23, kHdrFreqInc = 24, kHdrChannelBandwidth = 25,
    kHdrTimeStart = 26, kHdrTimeInc = 27, kHdrTimeAverage = 28,
    kHdrRefLon = 29, kHdrRefLat = 30, kHdrRefAlt = 31, kHdrStationX = 32,
    kHdrStationY = 33, kHdrStationZ = 34, kHdrElementX = 35,
    kHdrElementY = 36, kHdrElementZ = 37, kHdrStationName = 41,
    kHdrStationDiameter = 42, kHdrFeedAngleXA = 43
};
enum { kBlkDims = 1, kBlkAuto = 2, kBlkCross = 3, kBlkStationU = 7,
    kBlkStationV = 8, kBlkStationW = 9 };
// Polarisation types (binary_file.rst, "Visibility Polarisation Type").
enum { kPolStokesI = 1, kPolLinear = 10 };

// CRC-32C, byte-wise with a 256-entry table of the reflected polynomial.
struct Crc32c
{
    uint32_t table[256];
    Crc32c()
    {
        for (uint32_t i = 0; i < 256; ++i)
        {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k)
                c = (c & 1u) ? (c >> 1) ^ 0x82F63B78u : (c >> 1);
            table[i] = c;
        }
    }
    uint32_t update(uint32_t crc, const void* data, size_t n) const
    {
        const unsigned char* p = static_cast<const unsigned char*>(data);
        crc = ~crc;
        for (size_t i = 0; i < n; ++i)
            crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
        return ~crc;
    }
};

const Crc32c& crc32c()
{
    static const Crc32c c;
    return c;
}

size_t element_size(int type)
{
    size_t s = (type & kChar) ? 1 : (type & kInt) ? 4 : (type & kSingle) ? 4
            : (type & kDouble) ? 8 : 0;
    if (type & kComplex) s *= 2;
    if (type & kMatrix) s *= 4;
    return s;
}

void put_le(unsigned char* p, uint64_t v, int n)
{
    for (int i = 0; i < n; ++i) p[i] = (unsigned char) (v >> (8 * i));
}

}  // namespace
}  // namespace oskb

struct oskb_VisFile
{
    FILE* f;
    int amp_type, coord_type, num_stations, write_auto, write_cross;
    int error;
};

namespace oskb {
namespace {

// One chunk: tag, payload, CRC. Returns 0 or OSKB_ERR_INVALID_ARGUMENT /
// OSKB_ERR_MEMORY_COPY_FAILURE (write error).
int write_chunk(oskb_VisFile* h, int type, int group, int tag, int index,
        const void* data, size_t bytes)
{
    if (h->error) return h->error;
    const size_t es = element_size(type);
    if (es == 0 || es > 255) return OSKB_ERR_INVALID_ARGUMENT;
    unsigned char t[20];
    t[0] = 'T';
    t[1] = 0x40 + 2;
    t[2] = 'G';
    t[3] = (unsigned char) es;
    t[4] = 1u << 6;  // CRC present, little endian, standard tag
    t[5] = (unsigned char) type;
    t[6] = (unsigned char) group;
    t[7] = (unsigned char) tag;
    put_le(t + 8, (uint32_t) index, 4);
    put_le(t + 12, (uint64_t) bytes + 4, 8);
    uint32_t crc = crc32c().update(0, t, sizeof(t));
    if (bytes) crc = crc32c().update(crc, data, bytes);
    unsigned char c[4];
    put_le(c, crc, 4);
    if (fwrite(t, 1, sizeof(t), h->f) != sizeof(t) ||
            (bytes && fwrite(data, 1, bytes, h->f) != bytes) ||
            fwrite(c, 1, 4, h->f) != 4)
    {
        set_last_error_msg("vis file: write failed");
        h->error = OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    return h->error;
}

int write_int(oskb_VisFile* h, int group, int tag, int index, int v)
{
    int32_t x = v;
    return write_chunk(h, kInt, group, tag, index, &x, 4);
}

int write_double(oskb_VisFile* h, int group, int tag, int index, double v)
{
    return write_chunk(h, kDouble, group, tag, index, &v, 8);
}

int write_string(oskb_VisFile* h, int group, int tag, int index,
        const char* s)
{
    return write_chunk(h, kChar, group, tag, index, s, strlen(s) + 1);
}

}  // namespace
}  // namespace oskb

using namespace oskb;

extern "C" {

oskb_VisFile* oskb_vis_file_create(const char* filename, int amp_type,
        int coord_precision, int max_times_per_block, int num_times_total,
        int max_channels_per_block, int num_channels_total,
        int num_stations, int write_autocorr, int write_crosscorr,
        int casa_phase_convention, double freq_start_hz, double freq_inc_hz,
        double channel_bandwidth_hz, double time_start_mjd_utc,
        double time_inc_sec, double time_average_sec,
        int phase_centre_coord_type, double phase_centre_lon_deg,
        double phase_centre_lat_deg, double telescope_lon_deg,
        double telescope_lat_deg, double telescope_alt_m,
        const void* station_x, const void* station_y, const void* station_z,
        const double* station_diameter_m, const char* const* station_names,
        const int* num_elements, const void* element_x,
        const void* element_y, const void* element_z,
        const double* element_feed_angles, const char* telescope_path,
        const char* settings, const char* date_time, const char* version,
        const char* cwd, const char* username, int* status)
{
    if (*status) return nullptr;
    const int base = amp_type & 0x0F;
    if (!filename || !(amp_type & kComplex) || (base != kSingle &&
            base != kDouble) || (amp_type & ~(0x0F | kComplex | kMatrix)) ||
            (coord_precision != kSingle && coord_precision != kDouble) ||
            num_stations < 0 || num_times_total < 0 ||
            num_channels_total < 0 || (num_stations > 0 && (!station_x ||
            !station_y || !station_z)))
    {
        *status = OSKB_ERR_INVALID_ARGUMENT;
        return nullptr;
    }
    FILE* f = fopen(filename, "wb");
    if (!f)
    {
        set_last_error_msg("vis file: cannot open for writing");
        *status = OSKB_ERR_INVALID_ARGUMENT;
        return nullptr;
    }
    oskb_VisFile* h = (oskb_VisFile*) calloc(1, sizeof(oskb_VisFile));
    h->f = f;
    h->amp_type = amp_type;
    h->coord_type = coord_precision;
    h->num_stations = num_stations;
    h->write_auto = write_autocorr != 0;
    h->write_cross = write_crosscorr != 0;
    // File header: "OSKARBIN", NUL, version 2, 54 reserved zero bytes.
    unsigned char fh[64];
    memset(fh, 0, sizeof(fh));
    memcpy(fh, "OSKARBIN", 8);
    fh[9] = 2;
    if (fwrite(fh, 1, sizeof(fh), f) != sizeof(fh))
        h->error = OSKB_ERR_MEMORY_COPY_FAILURE;

    // ---- metadata (oskar_vis_header_write.c:40-87)
    char now[80];
    if (!date_time)
    {
        const time_t t = time(0);
        (void) strftime(now, sizeof(now), "%Y-%m-%d, %H:%M:%S (%Z)",
                localtime(&t));
        date_time = now;
    }
    write_string(h, kGroupMetadata, kMetaDateTime, 0, date_time);
    write_string(h, kGroupMetadata, kMetaVersion, 0,
            version ? version : oskb_version());
    std::string cwd_buf;
    if (!cwd)
    {
        char buf[4096];
        if (getcwd(buf, sizeof(buf))) cwd_buf = buf;
        if (!cwd_buf.empty()) cwd = cwd_buf.c_str();
    }
    if (cwd) write_string(h, kGroupMetadata, kMetaCwd, 0, cwd);
    if (!username)
    {
        username = getenv("USERNAME");
        if (!username) username = getenv("USER");
    }
    if (username && strlen(username) > 0)
        write_string(h, kGroupMetadata, kMetaUsername, 0, username);
    if (settings && strlen(settings) > 0)  // file contents, no NUL
        write_chunk(h, kChar, kGroupSettings, kSettingsContents, 0, settings,
                strlen(settings));

    // ---- dimensions and metadata (oskar_vis_header_write.c:89-199)
    const int g = kGroupVisHeader;
    write_chunk(h, kChar, g, kHdrTelescopePath, 0, telescope_path,
            telescope_path ? strlen(telescope_path) + 1 : 0);
    const int tags_per_block = 1 + (h->write_cross ? 4 : 0) +
            (h->write_auto ? 1 : 0);
    if (max_times_per_block <= 0) max_times_per_block = num_times_total;
    if (max_channels_per_block <= 0)
        max_channels_per_block = num_channels_total;
    write_int(h, g, kHdrTagsPerBlock, 0, tags_per_block);
    write_int(h, g, kHdrWriteAuto, 0, write_autocorr);
    write_int(h, g, kHdrWriteCross, 0, write_crosscorr);
    write_int(h, g, kHdrAmpType, 0, amp_type);
    write_int(h, g, kHdrCoordPrecision, 0, coord_precision);
    write_int(h, g, kHdrMaxTimes, 0, max_times_per_block);
    write_int(h, g, kHdrNumTimes, 0, num_times_total);
    write_int(h, g, kHdrMaxChannels, 0, max_channels_per_block);
    write_int(h, g, kHdrNumChannels, 0, num_channels_total);
    write_int(h, g, kHdrNumStations, 0, num_stations);
    write_int(h, g, kHdrPolType, 0, (amp_type & kMatrix) ? kPolLinear :
            kPolStokesI);
    write_int(h, g, kHdrCasa, 0, casa_phase_convention);
    write_int(h, g, kHdrPhaseCentreType, 0, phase_centre_coord_type);
    const double pc[2] = {phase_centre_lon_deg, phase_centre_lat_deg};
    write_chunk(h, kDouble, g, kHdrPhaseCentreDeg, 0, pc, sizeof(pc));
    write_double(h, g, kHdrFreqStart, 0, freq_start_hz);
    write_double(h, g, kHdrFreqInc, 0, freq_inc_hz);
    write_double(h, g, kHdrChannelBandwidth, 0, channel_bandwidth_hz);
    write_double(h, g, kHdrTimeStart, 0, time_start_mjd_utc);
    write_double(h, g, kHdrTimeInc, 0, time_inc_sec);
    write_double(h, g, kHdrTimeAverage, 0, time_average_sec);
    write_double(h, g, kHdrRefLon, 0, telescope_lon_deg);
    write_double(h, g, kHdrRefLat, 0, telescope_lat_deg);
    write_double(h, g, kHdrRefAlt, 0, telescope_alt_m);

    // ---- station and element coordinates (oskar_vis_header_write.c:
    // 201-219)
    const size_t cs = element_size(coord_precision);
    const size_t ns = (size_t) num_stations;
    write_chunk(h, coord_precision, g, kHdrStationX, 0, station_x, cs * ns);
    write_chunk(h, coord_precision, g, kHdrStationY, 0, station_y, cs * ns);
    write_chunk(h, coord_precision, g, kHdrStationZ, 0, station_z, cs * ns);
    size_t total_el = 0;
    for (int s = 0; s < num_stations; ++s)
        total_el += num_elements ? (size_t) num_elements[s] : 0;
    const unsigned char* ex = (const unsigned char*) element_x;
    const unsigned char* ey = (const unsigned char*) element_y;
    const unsigned char* ez = (const unsigned char*) element_z;
    size_t off = 0;
    for (int s = 0; s < num_stations; ++s)
    {
        const size_t n = num_elements ? (size_t) num_elements[s] : 0;
        const bool have = n && ex && ey && ez;
        write_chunk(h, coord_precision, g, kHdrElementX, s,
                have ? ex + cs * off : nullptr, have ? cs * n : 0);
        write_chunk(h, coord_precision, g, kHdrElementY, s,
                have ? ey + cs * off : nullptr, have ? cs * n : 0);
        write_chunk(h, coord_precision, g, kHdrElementZ, s,
                have ? ez + cs * off : nullptr, have ? cs * n : 0);
        off += n;
    }

    // ---- station names and diameters (oskar_vis_header_write.c:221-232)
    for (int s = 0; s < num_stations; ++s)
        write_string(h, g, kHdrStationName, s,
                station_names && station_names[s] ? station_names[s] : "");
    std::vector<double> diam(ns, 0.0);
    if (station_diameter_m)
        memcpy(diam.data(), station_diameter_m, sizeof(double) * ns);
    write_chunk(h, kDouble, g, kHdrStationDiameter, 0, diam.data(),
            sizeof(double) * ns);

    // ---- element feed angles, [feed X, Y][angle a, b, c][element]
    // (oskar_vis_header_write.c:234-251: tags 43-48 = X_A, Y_A, X_B, Y_B,
    // X_C, Y_C)
    off = 0;
    for (int s = 0; s < num_stations; ++s)
    {
        const size_t n = num_elements ? (size_t) num_elements[s] : 0;
        for (int angle = 0; angle < 3; ++angle)
            for (int feed = 0; feed < 2; ++feed)
            {
                const bool have = n && element_feed_angles;
                const double* a = have ? element_feed_angles +
                        (size_t) (3 * feed + angle) * total_el + off :
                        nullptr;
                write_chunk(h, kDouble, g, kHdrFeedAngleXA + 2 * angle +
                        feed, s, a, have ? sizeof(double) * n : 0);
            }
        off += n;
    }
    if (h->error)
    {
        *status = h->error;
        fclose(h->f);
        free(h);
        return nullptr;
    }
    return h;
}

int oskb_vis_file_write_block(oskb_VisFile* h, int block_index,
        int start_time_index, int start_channel_index, int num_times,
        int num_channels, const void* cross_correlations,
        const void* auto_correlations, const void* station_u,
        const void* station_v, const void* station_w)
{
    if (!h || block_index < 0 || num_times < 0 || num_channels < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (h->error) return h->error;
    const int N = h->num_stations;
    const int nbl = h->write_cross ? N * (N - 1) / 2 : 0;
    if ((h->write_cross && nbl > 0 && !cross_correlations) ||
            (h->write_auto && !auto_correlations))
        return OSKB_ERR_INVALID_ARGUMENT;
    // dimensions: start time, start channel, times, channels, baselines,
    // stations (oskar_vis_block_write.c:22-25)
    const int32_t dims[6] = {start_time_index, start_channel_index,
            num_times, num_channels, nbl, N};
    const int g = kGroupVisBlock;
    write_chunk(h, kInt, g, kBlkDims, block_index, dims, sizeof(dims));
    // arrays are written when they hold data, as the reference tests their
    // lengths (oskar_vis_block_accessors.c:55-68)
    const size_t es = element_size(h->amp_type);
    const size_t tc = (size_t) num_times * num_channels;
    if (h->write_auto && tc * N > 0)
        write_chunk(h, h->amp_type, g, kBlkAuto, block_index,
                auto_correlations, es * tc * N);
    if (h->write_cross && tc * nbl > 0)
    {
        write_chunk(h, h->amp_type, g, kBlkCross, block_index,
                cross_correlations, es * tc * nbl);
        if (station_u && station_v && station_w)
        {
            const size_t b = element_size(h->coord_type) * num_times * N;
            write_chunk(h, h->coord_type, g, kBlkStationU, block_index,
                    station_u, b);
            write_chunk(h, h->coord_type, g, kBlkStationV, block_index,
                    station_v, b);
            write_chunk(h, h->coord_type, g, kBlkStationW, block_index,
                    station_w, b);
        }
    }
    return h->error;
}

int oskb_vis_file_close(oskb_VisFile* h)
{
    if (!h) return OSKB_ERR_INVALID_ARGUMENT;
    int err = h->error;
    if (fclose(h->f) != 0 && !err) err = OSKB_ERR_MEMORY_COPY_FAILURE;
    free(h);
    return err;
}

}  // extern "C"
