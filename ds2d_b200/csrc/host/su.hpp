// Minimal Seismic Unix (SU) trace I/O for the DS2D host driver.
//
// An SU file is a sequence of traces, each a 240-byte SEG-Y trace header followed by ns float
// samples (native byte order).  Only the header words the reference reads are used
// (subfun/segy.h:8-309: sx at byte 72, gx at byte 80, ns at byte 114, dt in microseconds at
// byte 116; main.cpp:52-155 index_shot, :253-270 read_shot_gather_su).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace ds2d_host {

constexpr int kSuHeader = 240;

struct SuTrace {
  int32_t sx = 0, gx = 0;
  uint16_t ns = 0, dt_us = 0;
};

inline void su_decode(const unsigned char *h, SuTrace &t) {
  std::memcpy(&t.sx, h + 72, 4);
  std::memcpy(&t.gx, h + 80, 4);
  std::memcpy(&t.ns, h + 114, 2);
  std::memcpy(&t.dt_us, h + 116, 2);
}

inline void su_encode(unsigned char *h, const SuTrace &t, int tracl) {
  std::memset(h, 0, kSuHeader);
  std::memcpy(h + 0, &tracl, 4);
  std::memcpy(h + 72, &t.sx, 4);
  std::memcpy(h + 80, &t.gx, 4);
  std::memcpy(h + 114, &t.ns, 2);
  std::memcpy(h + 116, &t.dt_us, 2);
}

// One shot gather of the file: consecutive traces sharing sx (main.cpp:52-155 table row).
struct ShotIndex {
  int sno;        // 1-based shot number
  int ntr;        // traces
  int sx;         // source x coordinate
  int xmin, xmax; // aperture over source and receivers
  long long pos;  // index of the first trace
};

// Indexes the shots of an SU file; returns false (with a message) on a malformed file.
inline bool su_index(const std::string &path, int *nt, float *dt, std::vector<ShotIndex> &table,
                     std::string &err) {
  FILE *fp = std::fopen(path.c_str(), "rb");
  if (!fp) {
    err = "cannot open " + path;
    return false;
  }
  unsigned char h[kSuHeader];
  SuTrace t;
  table.clear();
  long long pos = 0;
  int sx0 = 0;
  bool first = true;
  *nt = 0;
  while (std::fread(h, 1, kSuHeader, fp) == (size_t)kSuHeader) {
    su_decode(h, t);
    if (first) {
      *nt = t.ns;
      *dt = t.dt_us / 1.0e6f;
      if (*nt <= 0) {
        err = path + ": first trace has ns = 0";
        std::fclose(fp);
        return false;
      }
    } else if (t.ns != *nt) {
      err = path + ": traces with different ns";
      std::fclose(fp);
      return false;
    }
    const int xmin = std::min(t.sx, t.gx), xmax = std::max(t.sx, t.gx);
    if (first || t.sx != sx0) {
      table.push_back(ShotIndex{(int)table.size() + 1, 0, t.sx, xmin, xmax, pos});
      sx0 = t.sx;
      first = false;
    }
    ShotIndex &s = table.back();
    s.ntr++;
    s.xmin = std::min(s.xmin, xmin);
    s.xmax = std::max(s.xmax, xmax);
    if (std::fseek(fp, (long)(*nt) * 4, SEEK_CUR) != 0) {
      err = path + ": truncated trace";
      std::fclose(fp);
      return false;
    }
    pos++;
  }
  std::fclose(fp);
  if (table.empty()) {
    err = path + ": no traces";
    return false;
  }
  return true;
}

// Reads ntr traces starting at trace `pos` (main.cpp:253-270): samples into dat[ntr][nt], the
// receiver coordinates into gx.
inline bool su_read_gather(const std::string &path, long long pos, int ntr, int nt, float *dat,
                           int *gx, std::string &err) {
  FILE *fp = std::fopen(path.c_str(), "rb");
  if (!fp) {
    err = "cannot open " + path;
    return false;
  }
  const long long tl = kSuHeader + 4LL * nt;
  if (std::fseek(fp, (long)(tl * pos), SEEK_SET) != 0) {
    err = path + ": seek failed";
    std::fclose(fp);
    return false;
  }
  unsigned char h[kSuHeader];
  SuTrace t;
  for (int i = 0; i < ntr; i++) {
    if (std::fread(h, 1, kSuHeader, fp) != (size_t)kSuHeader ||
        std::fread(dat + (size_t)i * nt, 4, nt, fp) != (size_t)nt) {
      err = path + ": truncated gather";
      std::fclose(fp);
      return false;
    }
    su_decode(h, t);
    gx[i] = t.gx;
  }
  std::fclose(fp);
  return true;
}

}  // namespace ds2d_host
