/* Stands in for the configure-generated header (mbx_version.h.in). */
#define MBX_VERSION "1.3.3"
