// Stand-in for the one OpenCV type the reference headers name (cv::Mat, as a
// parameter type only) so the reference kernels compile for the checker
// without OpenCV.  Nothing here is called.
#pragma once
namespace cv {
class Mat {
public:
    template <class T>
    T& at(int, int);
    bool empty() const { return true; }
    unsigned char* data = nullptr;
};
}  // namespace cv
