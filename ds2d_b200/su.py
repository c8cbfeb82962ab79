"""Seismic Unix (SU) trace files: 240-byte SEG-Y trace headers + float samples (native order).

Only the header words the reference reads are written (subfun/segy.h: sx at byte 72, gx at
byte 80, ns at byte 114, dt in microseconds at byte 116)."""
import numpy as np

HEADER = 240


def write_su(path, data, sx, gx, dt):
    """data [ntr][ns] float32; sx, gx per trace (ints); dt in seconds."""
    data = np.ascontiguousarray(data, np.float32)
    ntr, ns = data.shape
    with open(path, "wb") as f:
        for i in range(ntr):
            h = np.zeros(HEADER, np.uint8)
            h[0:4] = np.frombuffer(np.int32(i + 1).tobytes(), np.uint8)
            h[72:76] = np.frombuffer(np.int32(sx[i]).tobytes(), np.uint8)
            h[80:84] = np.frombuffer(np.int32(gx[i]).tobytes(), np.uint8)
            h[114:116] = np.frombuffer(np.uint16(ns).tobytes(), np.uint8)
            h[116:118] = np.frombuffer(np.uint16(round(dt * 1e6)).tobytes(), np.uint8)
            f.write(h.tobytes())
            f.write(data[i].tobytes())


def read_su(path):
    """Returns (data [ntr][ns], sx, gx, dt)."""
    raw = open(path, "rb").read()
    ns = int(np.frombuffer(raw[114:116], np.uint16)[0])
    dt = int(np.frombuffer(raw[116:118], np.uint16)[0]) / 1e6
    tl = HEADER + 4 * ns
    ntr = len(raw) // tl
    buf = np.frombuffer(raw[:ntr * tl], np.uint8).reshape(ntr, tl)
    sx = buf[:, 72:76].copy().view(np.int32).ravel()
    gx = buf[:, 80:84].copy().view(np.int32).ravel()
    data = buf[:, HEADER:].copy().view(np.float32)
    return data, sx, gx, dt
