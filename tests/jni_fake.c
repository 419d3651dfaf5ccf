/* A fake JNIEnv for tests: the JNI functions libGPUALS.so's Spark shim calls,
 * installed at their slots of the JNI specification's interface function
 * table, over plain heap arrays. Test infrastructure only. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { int kind; int len; void *data; } jarr; /* kind: 0 object, 1 int, 2 float */

static void *table[240];
static void *env_ptr = table;
static int live_critical = 0;

static void *FindClass(void *env, const char *name) { (void)env; (void)name; return (void *)0x1; }
static void DeleteLocalRef(void *env, void *o) { (void)env; (void)o; }
static int frames = 0, max_frames = 0;
static int PushLocalFrame(void *env, int capacity) {
  (void)env; (void)capacity; if (++frames > max_frames) max_frames = frames; return 0;
}
static void *PopLocalFrame(void *env, void *result) { (void)env; --frames; return result; }
static int GetArrayLength(void *env, jarr *a) { (void)env; return a->len; }
static jarr *new_arr(int kind, int len, size_t elem) {
  jarr *a = (jarr *)calloc(1, sizeof(jarr));
  a->kind = kind; a->len = len; a->data = calloc((size_t)(len > 0 ? len : 1), elem);
  return a;
}
static jarr *NewObjectArray(void *env, int len, void *cls, void *init) {
  (void)env; (void)cls; (void)init; return new_arr(0, len, sizeof(void *));
}
static void *GetObjectArrayElement(void *env, jarr *a, int i) { (void)env; return ((void **)a->data)[i]; }
static void SetObjectArrayElement(void *env, jarr *a, int i, void *v) { (void)env; ((void **)a->data)[i] = v; }
static jarr *NewFloatArray(void *env, int len) { (void)env; return new_arr(2, len, sizeof(float)); }
static void GetFloatArrayRegion(void *env, jarr *a, int start, int len, float *buf) {
  (void)env; memcpy(buf, (float *)a->data + start, sizeof(float) * (size_t)len);
}
static void SetFloatArrayRegion(void *env, jarr *a, int start, int len, const float *buf) {
  (void)env; memcpy((float *)a->data + start, buf, sizeof(float) * (size_t)len);
}
static void *GetPrimitiveArrayCritical(void *env, jarr *a, uint8_t *copy) {
  (void)env; if (copy) *copy = 0; ++live_critical; return a->data;
}
static void ReleasePrimitiveArrayCritical(void *env, jarr *a, void *p, int mode) {
  (void)env; (void)a; (void)p; (void)mode; --live_critical;
}

void *fake_env(void) {
  table[6] = (void *)FindClass;
  table[19] = (void *)PushLocalFrame;
  table[20] = (void *)PopLocalFrame;
  table[23] = (void *)DeleteLocalRef;
  table[171] = (void *)GetArrayLength;
  table[172] = (void *)NewObjectArray;
  table[173] = (void *)GetObjectArrayElement;
  table[174] = (void *)SetObjectArrayElement;
  table[181] = (void *)NewFloatArray;
  table[205] = (void *)GetFloatArrayRegion;
  table[213] = (void *)SetFloatArrayRegion;
  table[222] = (void *)GetPrimitiveArrayCritical;
  table[223] = (void *)ReleasePrimitiveArrayCritical;
  return &env_ptr;
}
void *fake_float_array(int len, const float *src) {
  jarr *a = new_arr(2, len, sizeof(float));
  if (src) memcpy(a->data, src, sizeof(float) * (size_t)len);
  return a;
}
void *fake_int_array(int len, const int *src) {
  jarr *a = new_arr(1, len, sizeof(int));
  if (src) memcpy(a->data, src, sizeof(int) * (size_t)len);
  return a;
}
void *fake_object_array(int len) { return new_arr(0, len, sizeof(void *)); }
void fake_set(jarr *a, int i, void *v) { ((void **)a->data)[i] = v; }
int fake_length(jarr *a) { return a->len; }
void *fake_get(jarr *a, int i) { return ((void **)a->data)[i]; }
float *fake_float_data(jarr *a) { return (float *)a->data; }
int fake_live_critical(void) { return live_critical; }
int fake_open_frames(void) { return frames; }
int fake_max_frames(void) { return max_frames; }
