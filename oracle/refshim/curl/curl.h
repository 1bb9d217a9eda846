/* Stand-in for libcurl's header.  The reference uses curl only to download
 * residue tables (source/core/utility/Curl.cpp:13-58), which the oracle never
 * calls; every function here reports failure. */
#pragma once
typedef void CURL;
typedef int CURLcode;
typedef int CURLoption;
#define CURLE_OK 0
#define CURL_GLOBAL_DEFAULT 3
#define CURLOPT_URL 10002
#define CURLOPT_WRITEDATA 10001
static inline CURLcode curl_global_init(long) { return 1; }
static inline void curl_global_cleanup(void) {}
static inline const char* curl_easy_strerror(CURLcode) { return "curl unavailable in the oracle build"; }
static inline CURL* curl_easy_init(void) { return 0; }
static inline void curl_easy_cleanup(CURL*) {}
template <typename T> static inline CURLcode curl_easy_setopt(CURL*, CURLoption, T) { return 1; }
static inline CURLcode curl_easy_perform(CURL*) { return 1; }
