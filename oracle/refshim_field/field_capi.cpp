// field_capi.cpp -- ORACLE (test infrastructure only).
//
// Drives the reference's CMS field-map reader (examples/magneticfield/
// simplifiedCMS/inc/Geant/ScalarCMSmagField.h) compiled in place through the
// shims in this directory, to pin the library's field-map lookup.  Built into
// its own library (oracle/_ref/libgxref_field.so).
#include "Geant/ScalarCMSmagField.h"

static ScalarCMSmagField *g_field = nullptr;

extern "C" {

int gxref_field_load(const char *path)
{
  delete g_field;
  g_field = new ScalarCMSmagField(path);
  return 1;
}

// field (tesla) at n points (mm)
void gxref_field_value(int n, const double *pos, double *B)
{
  for (int i = 0; i < n; ++i) {
    vecgeom::Vector3D<double> p(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), b;
    g_field->GetFieldValue(p, b);
    B[3 * i] = b.x();
    B[3 * i + 1] = b.y();
    B[3 * i + 2] = b.z();
  }
}

} // extern "C"
