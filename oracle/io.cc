// Oracle (test infrastructure): wavy-surface output layouts.
#include "oracle.h"

#include <cstring>
#include <fstream>

// Reference: src/io/binary_stream.hh:43-60 with src/bits/byte_swap.hh: raw
// values of the surface in C order (t slowest), each in network byte order.
extern "C" int orc_write_zeta_bin(const char* path, const double* zeta, size_t n) {
	std::ofstream out(path, std::ios::binary);
	if (!out) return -1;
	for (size_t i = 0; i < n; ++i) {
		unsigned char b[8];
		std::memcpy(b, &zeta[i], 8);
		for (int k = 0; k < 4; ++k) { unsigned char t = b[k]; b[k] = b[7 - k]; b[7 - k] = t; }
		out.write(reinterpret_cast<const char*>(b), 8);
	}
	return out ? 0 : -2;
}

// Reference: src/bits/write_csv.hh:13-42: header "t,x,y,z"; t is the slice
// index, x and y are grid coordinates; default ostream precision.
extern "C" int orc_write_zeta_csv(const char* path, const double* zeta, int nt,
                                  int nx, int ny, const double delta[3]) {
	std::ofstream out(path);
	if (!out) return -1;
	out << 't' << ',' << 'x' << ',' << 'y' << ',' << 'z' << '\n';
	for (int i = 0; i < nt; ++i)
		for (int j = 0; j < nx; ++j)
			for (int k = 0; k < ny; ++k) {
				const double x = delta[1] * j;
				const double y = delta[2] * k;
				out << i << ',' << x << ',' << y << ',' << zeta[(size_t(i) * nx + j) * ny + k] << '\n';
			}
	return out ? 0 : -2;
}
