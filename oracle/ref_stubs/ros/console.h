// TEST INFRASTRUCTURE -- stand-in for ros/console.h: the logging macros print to stderr.
#pragma once
#include <cstdio>
#define ROS_WARN(...) (std::fprintf(stderr, __VA_ARGS__), std::fputc('\n', stderr))
#define ROS_INFO(...) (std::fprintf(stderr, __VA_ARGS__), std::fputc('\n', stderr))
#define ROS_ERROR(...) (std::fprintf(stderr, __VA_ARGS__), std::fputc('\n', stderr))
#define ROS_DEBUG(...) ((void)0)
